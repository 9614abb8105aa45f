"""GPU test of sclbm_mass_momentum_noalloc, the monitor for callers that may
not allocate device memory (a host that owns all device memory through a
fixed arena, or code that runs where cudaMalloc is not allowed).

The caller owns every buffer: here torch allocates the populations and the
mask on the device, never the library.  The entry point must agree with the
allocating monitor (sclbm_domain_mass_momentum) on the same state, within the
tolerance of the monitor tests, on two calls in a row -- the second call sees
the scratch array exactly as the first left it.  This file sorts last so a
run that stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import cases
import gpu_runner

pytestmark = pytest.mark.gpu

W = cases.W
RUNS = cases.all_cases()


def _device_buffers(torch, dom, prec, rho_ref, mask):
    """Populations in the domain's storage form, in caller-owned device memory."""
    dtype = {0: np.float64, 1: np.float32, 2: np.float16}[prec]
    out = []
    for k in range(dom.ncomp):
        f = dom.download_f(k).reshape(9, -1)
        if prec != 0:
            f = f - W[:, None] * rho_ref[k]   # exact inverse of the download shift
            f[:, mask == 0] = 0.0
        out.append(torch.from_numpy(np.ascontiguousarray(f.astype(dtype)).ravel()).cuda())
    return out


def _noalloc(sc, bufs, mask_dev, nx, ny, ncomp, prec, rho_ref, stream):
    from sc_lbm_b200 import capi
    out = np.zeros(7)
    rr = (C.c_double * 2)(*rho_ref)
    f1 = bufs[1].data_ptr() if ncomp > 1 else None
    rc = capi.lib().sclbm_mass_momentum_noalloc(
        C.c_void_p(bufs[0].data_ptr()), C.c_void_p(f1) if f1 else None,
        C.c_void_p(mask_dev.data_ptr()), nx, ny, ncomp, prec, rr, C.c_void_p(stream),
        out.ctypes.data_as(C.POINTER(C.c_double)))
    capi.check(rc)
    return out


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_noalloc_monitor_matches_allocating_monitor(sclbm, prec):
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream().cuda_stream
    for name, rr in (("channel_80x32", (0.6, 1.4)), ("spinodal_48x40", (1.0, 1.0))):
        case = RUNS[name]
        dom = gpu_runner.make_domain(sclbm, case, prec, rho_ref=rr)
        mask = np.asarray(gpu_runner._geometry(sclbm, case)[1], np.uint8)
        mask_dev = torch.from_numpy(mask.copy()).cuda()
        for call in range(2):  # two calls in a row, the state advanced in between
            dom.step(7 + call)
            want = dom.mass_momentum()
            bufs = _device_buffers(torch, dom, prec, rr, mask)
            got = _noalloc(sclbm, bufs, mask_dev, case["nx"], case["ny"], 2, prec, rr, stream)
            torch.cuda.synchronize()
            for k in range(2):
                assert np.isclose(got[3 * k], want[3 * k], rtol=1e-12), (name, prec, call, k)
                for v in (1, 2):
                    assert np.isclose(got[3 * k + v], want[3 * k + v], rtol=1e-9, atol=1e-9)
            assert got[6] == 0


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_noalloc_monitor_single_component(sclbm, prec):
    """One component (the Poiseuille channel of the measurement plan): the
    second population pointer is unused and only out[0..2] carry sums."""
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream().cuda_stream
    case = RUNS["poiseuille_200x50"]
    rr = (1.0, 0.0)
    dom = gpu_runner.make_domain(sclbm, case, prec, rho_ref=rr)
    mask = np.asarray(gpu_runner._geometry(sclbm, case)[1], np.uint8)
    mask_dev = torch.from_numpy(mask.copy()).cuda()
    for call in range(2):
        dom.step(11 + call)
        want = dom.mass_momentum()
        bufs = _device_buffers(torch, dom, prec, rr, mask)
        got = _noalloc(sclbm, bufs, mask_dev, case["nx"], case["ny"], 1, prec, rr, stream)
        torch.cuda.synchronize()
        assert np.isclose(got[0], want[0], rtol=1e-12), (prec, call)
        for v in (1, 2):
            assert np.isclose(got[v], want[v], rtol=1e-9, atol=1e-12), (prec, call, v)
        assert np.all(got[3:6] == 0.0) and got[6] == 0


def test_noalloc_monitor_reports_non_finite_populations(sclbm):
    """A NaN planted in the caller's buffer (plain data written from the host)
    is counted and returned as SCLBM_E_NONFINITE; the next clean call is ok."""
    torch = pytest.importorskip("torch")
    from sc_lbm_b200 import capi
    stream = torch.cuda.current_stream().cuda_stream
    case = RUNS["channel_80x32"]
    rr = (0.6, 1.4)
    dom = gpu_runner.make_domain(sclbm, case, 0, rho_ref=rr)
    dom.step(3)
    mask = np.asarray(gpu_runner._geometry(sclbm, case)[1], np.uint8)
    mask_dev = torch.from_numpy(mask.copy()).cuda()
    bufs = _device_buffers(torch, dom, 0, rr, mask)
    node = int(np.flatnonzero(mask)[17])
    N = case["nx"] * case["ny"]
    bufs[1][4 * N + node] = float("nan")
    out = np.zeros(7)
    r2 = (C.c_double * 2)(*rr)
    rc = capi.lib().sclbm_mass_momentum_noalloc(
        C.c_void_p(bufs[0].data_ptr()), C.c_void_p(bufs[1].data_ptr()),
        C.c_void_p(mask_dev.data_ptr()), case["nx"], case["ny"], 2, 0, r2, C.c_void_p(stream),
        out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == capi.E_NONFINITE
    assert out[6] == 1.0
    bufs[1][4 * N + node] = 0.0
    got = _noalloc(sclbm, bufs, mask_dev, case["nx"], case["ny"], 2, 0, rr, stream)
    assert got[6] == 0


def test_noalloc_monitor_refuses_a_capturing_stream(sclbm):
    """It synchronises its stream to return the sums, so a stream under graph
    capture is refused before anything is enqueued and the capture survives."""
    torch = pytest.importorskip("torch")
    from sc_lbm_b200 import capi
    case = RUNS["spinodal_48x40"]
    dom = gpu_runner.make_domain(sclbm, case, 0)
    mask = np.asarray(gpu_runner._geometry(sclbm, case)[1], np.uint8)
    mask_dev = torch.from_numpy(mask.copy()).cuda()
    bufs = _device_buffers(torch, dom, 0, (1.0, 1.0), mask)
    side = torch.cuda.Stream()
    # warm-up call outside the capture: address lookup and kernel loading
    _noalloc(sclbm, bufs, mask_dev, case["nx"], case["ny"], 2, 0, (1.0, 1.0), side.cuda_stream)
    x = torch.ones(64, device="cuda")
    g = torch.cuda.CUDAGraph()
    out = np.zeros(7)
    with torch.cuda.stream(side):
        g.capture_begin()
        y = x * 2.0
        rc = capi.lib().sclbm_mass_momentum_noalloc(
            C.c_void_p(bufs[0].data_ptr()), C.c_void_p(bufs[1].data_ptr()),
            C.c_void_p(mask_dev.data_ptr()), case["nx"], case["ny"], 2, 0, None,
            C.c_void_p(side.cuda_stream), out.ctypes.data_as(C.POINTER(C.c_double)))
        g.capture_end()
    assert rc == capi.E_INVALID_ARGUMENT
    assert "captured" in capi.last_error()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(y, torch.full_like(x, 2.0))


def test_noalloc_monitor_rejects_oversized_lattices(sclbm):
    torch = pytest.importorskip("torch")
    from sc_lbm_b200 import capi
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    m = torch.ones(16, dtype=torch.uint8, device="cuda")
    out = np.zeros(7)
    # 16384 x 16384 = 2^28 nodes: beyond the fixed scratch; refused before any launch
    rc = capi.lib().sclbm_mass_momentum_noalloc(
        C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), C.c_void_p(m.data_ptr()),
        16384, 16384, 2, 0, None, None, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == capi.E_INVALID_ARGUMENT
    assert "too large" in capi.last_error()
    # nx * ny wraps around 2^64 to a small product: refused all the same
    rc = capi.lib().sclbm_mass_momentum_noalloc(
        C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), C.c_void_p(m.data_ptr()),
        1 << 40, 1 << 30, 2, 0, None, None, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == capi.E_INVALID_ARGUMENT
    assert "too large" in capi.last_error()
