// petscts.h -- TEST INFRASTRUCTURE ONLY: forwards to the DMDA layer of the oracle's
// reference build.
#pragma once
#include "petscdmda.h"
