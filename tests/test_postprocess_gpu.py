"""GPU post-processing (langevina_b200.postprocess over lgv_x2k,
lgv_x2k_rotated, lgv_time_correlator) against the reference and the oracle:

- the time correlators reproduce the reference's own Loader.py outputs
  (tests/golden/otot.json) and the oracle on many series at once, real and
  complex, ragged series counts, decimation, connected part, lags up to T - 1;
- x2k of a measured wall is the measurer's k wall bit for bit, and matches the
  oracle on arbitrary rows;
- x2k_rotated matches the oracle and the measurer's rotated k walls;
- a device-resident measurement history goes through x2k-ordered k walls into
  computeOtOtp(d, conj(d)) without leaving the GPU.
"""
import ctypes as C

import numpy as np
import pytest

import postprocess as P  # oracle/postprocess.py (test infrastructure)
from lgvtest import GpuLattice, rand_state
from test_postprocess_oracle import case_inputs, dec, golden_cases, golden_series, run_case

pytestmark = pytest.mark.gpu

HB = 4


def close(got, want, rtol=1e-12):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape, (got.shape, want.shape)
    scale = max(1.0, float(np.max(np.abs(want)))) if want.size else 1.0
    err = float(np.max(np.abs(got - want))) if want.size else 0.0
    assert err <= rtol * scale, f"max error {err:.3e} (scale {scale:.3e})"


@pytest.mark.parametrize("i", range(10))
def test_correlators_match_reference_loader(lgv, i):
    from langevina_b200 import postprocess as G

    c = golden_cases()[i]
    x, y = case_inputs(c, golden_series())
    close(run_case(G, c, x, y), dec(c["out"]))


@pytest.mark.parametrize("T,ns,cplx,decim,conn,ntmax", [
    (1, 1, False, 1, False, 1), (2, 3, True, 1, True, 2), (17, 33, False, 1, False, 17),
    (40, 70, True, 1, True, 23), (300, 70, False, 1, True, 129), (300, 5, True, 2, False, 300),
    (257, 64, True, 5, True, 40), (64, 31, False, 3, False, 64), (1000, 129, True, 1, False, 200)])
def test_correlators_many_series_match_oracle(lgv, T, ns, cplx, decim, conn, ntmax):
    from langevina_b200 import postprocess as G

    rng = np.random.default_rng(T * 1000 + ns)
    a = rng.normal(size=(T, ns)) + 0.2
    b = rng.normal(size=(T, ns)) - 0.1
    if cplx:
        a = a + 1j * rng.normal(size=(T, ns))
        b = b + 1j * rng.normal(size=(T, ns))
    got, err = G.computeOtOtp(a, b, conn=conn, nTMax=ntmax, decim=decim)
    want, _ = P.computeOtOtp(a, b, conn=conn, nTMax=ntmax, decim=decim)
    close(got, want)
    assert not np.any(err)


def test_correlator_trailing_dims_and_torch_in_place(lgv):
    import torch
    from langevina_b200 import postprocess as G

    rng = np.random.default_rng(5)
    a = rng.normal(size=(120, 3, 11, 9)) + 1j * rng.normal(size=(120, 3, 11, 9))
    ta = torch.from_numpy(a).cuda()
    got, _ = G.computeOtOtp(ta, torch.conj(ta).resolve_conj(), nTMax=30)
    assert isinstance(got, torch.Tensor) and got.is_cuda and got.shape == (30, 3, 11, 9)
    want, _ = P.computeOtOtp(a, np.conj(a), nTMax=30)
    close(got.cpu().numpy(), want)


def test_correlator_errors(lgv):
    from langevina_b200 import _lib as L
    from langevina_b200 import postprocess as G

    a = np.ones((10, 2))
    with pytest.raises(ValueError):
        G.computeOtOtp(a, a, nTMax=11)
    with pytest.raises(NotImplementedError):
        G.computeOtOtp(a, a, statFunc=lambda x: (np.median(x), 0))
    lib = L.load()
    dummy = C.c_void_p(16)
    assert lib.lgv_time_correlator(dummy, dummy, 10, 2, 2, 0, 0, 1, 0, dummy, None) == L.LGV_ERR_INVALID
    assert lib.lgv_time_correlator(dummy, dummy, 10, 2, 1, 0, 5, 1, 0, dummy, None) == L.LGV_ERR_INVALID
    assert lib.lgv_x2k(dummy, 1, 7, dummy, None) == L.LGV_ERR_INVALID


def test_x2k_matches_oracle(lgv):
    from langevina_b200 import postprocess as G

    rng = np.random.default_rng(6)
    for N in (2, 8, 34, 256, 512, 1000):  # 512: largest tiled size; 1000: one thread per (row, k)
        w = rng.normal(size=(7, 3, N))
        close(G.x2k(w), P.x2k(w), rtol=1e-13)


def test_x2k_rotated_matches_oracle(lgv):
    from langevina_b200 import postprocess as G

    rng = np.random.default_rng(7)
    wk = rng.normal(size=(4, 14, 9, 2))
    wk[1, 0:4, 0, :] = 0.0
    close(G.x2k_rotated(wk), P.x2k_rotated(wk), rtol=1e-13)


def test_transforms_reproduce_the_measurer(lgv):
    from langevina_b200 import postprocess as G

    N = 16
    g = GpuLattice(lgv, N, mass0=-4.813, lam=10.0, H=0.01, seed=9)
    g.set_state(rand_state(N, 9, phi_scale=0.7))
    g.step(HB, 0.1, nsteps=5)
    m = g.measure()
    for a in range(3):
        assert np.array_equal(G.x2k(m.wall[a]), m.wall_k[a]), f"axis {a}"
        assert np.array_equal(G.x2k(m.wall_phase[a]), m.wall_phase_k[a]), f"phase axis {a}"
        rot = G.x2k_rotated(m.wall_k[a][None])[0]
        close(rot, m.wall_k_rotated[a][:13], rtol=1e-14)
    g.close()


def test_device_history_correlator(lgv):
    import torch
    from langevina_b200 import postprocess as G

    N, T = 16, 200
    NK = N // 2 + 1
    g = GpuLattice(lgv, N, mass0=-4.813, lam=10.0, H=0.01, seed=10)
    g.initialize(1, 0.3)
    stream = torch.cuda.current_stream()
    g.L.check(g.lib.lgv_set_stream(g.h, C.c_void_p(stream.cuda_stream)), "set_stream")
    size = int(g.lib.lgv_measure_size(N))
    hist = torch.empty((T, size), dtype=torch.float64, device="cuda")
    for t in range(T):
        g.step(HB, 0.1, nsteps=2)
        g.L.check(g.lib.lgv_measure_device(g.h, C.c_void_p(hist[t].data_ptr())), "measure_device")
    lo = 11 + 33 * N  # wall_k of the x axis in the packed measurement
    wk = hist[:, lo:lo + 11 * NK * 2].reshape(T, 11, NK, 2)
    d = torch.view_as_complex(wk.contiguous())
    got, _ = G.computeOtOtp(d, torch.conj(d).resolve_conj(), nTMax=50, conn=True)
    dn = d.cpu().numpy()
    want, _ = P.computeOtOtp(dn, np.conj(dn), nTMax=50, conn=True)
    close(got.cpu().numpy(), want)
    g.close()


def test_correlator_unaligned_complex_pairs(lgv):
    """Complex series whose pairs do not start on 16 bytes (an 8-byte offset
    into the buffer) take the kernel's two-load path; same results."""
    import torch
    from langevina_b200 import _lib as L

    T, ns, ntmax = 90, 37, 31
    rng = np.random.default_rng(8)
    a = rng.normal(size=(T, ns)) + 1j * rng.normal(size=(T, ns))
    b = rng.normal(size=(T, ns)) + 1j * rng.normal(size=(T, ns))
    bufs = []
    for x in (a, b):
        t = torch.zeros(T * ns * 2 + 1, dtype=torch.float64, device="cuda")
        t[1:].copy_(torch.from_numpy(np.ascontiguousarray(x).view(np.float64).ravel()))
        bufs.append(t)
    out = torch.zeros(ntmax * ns * 2 + 1, dtype=torch.float64, device="cuda")
    lib = L.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    L.check(lib.lgv_time_correlator(C.c_void_p(bufs[0].data_ptr() + 8), C.c_void_p(bufs[1].data_ptr() + 8), T, ns,
                                    2 * ns, 1, ntmax, 1, 1, C.c_void_p(out.data_ptr() + 8), stream),
            "lgv_time_correlator")
    got = out[1:].cpu().numpy().view(np.complex128).reshape(ntmax, ns)
    want, _ = P.computeOtOtp(a, b, conn=True, nTMax=ntmax)
    close(got, want)
