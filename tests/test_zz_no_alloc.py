"""apo_pme_reciprocal_static (the reciprocal-space entry point that uses a
static device scratch area instead of allocations) against the context's
reciprocal part, the existing entry point for the same kernels.

Collected last on purpose: it must pass after every other GPU test has run
in the same process, as well as alone.
"""
import ctypes

import numpy as np
import pytest

from apocharmm_b200 import api
from apocharmm_b200._lib import lib
from apocharmm_b200.systems import water_box
from parity_util import oracle_for

pytestmark = pytest.mark.gpu

FORCE_SCALE = 2.0 ** 40
# Same kernels; the context spreads from cluster-local single-precision
# coordinates plus the cluster origin, this entry point from plain absolute
# single-precision coordinates, so the two differ by coordinate rounding only.
FORCE_RTOL = 1e-5
ENERGY_RTOL = 1e-6


def _static_call(torch, xyzq, n, box, nfft, order, kappa, grad, stride, energy, fp64):
    fn = lib().apo_pme_reciprocal_static
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                   ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                   ctypes.c_int, ctypes.c_void_p]
    st = fn(xyzq, n, box[0], box[1], box[2], nfft[0], nfft[1], nfft[2], order, kappa, grad,
            stride, energy, int(fp64), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st


@pytest.mark.parametrize("order,nfft,precise", [(4, (24, 24, 24), False),
                                                 (6, (28, 30, 32), True)])
def test_static_reciprocal_matches_context(tmp_path, order, nfft, precise):
    torch = pytest.importorskip("torch")
    s = water_box(512, 25.0, seed=11)
    settings = dict(kappa=0.34, nfft=nfft, order=order, ctofnb=10.0, ctonnb=8.0, cutnb=12.0)
    psf, prm, fm, ctx = api.system_context(s, str(tmp_path), precise=precise, settings=settings)
    fm.setComponentMask(4)
    ctx.calculateForces(False, True, False)
    G_ref = ctx.getForces()
    E = ctx.getEnergyComponents()
    ewks_ref = E["ewks"]

    n = s.n_atoms
    x = ctx.getCoordinates()
    xyzq_h = np.zeros((n, 4), np.float32)
    xyzq_h[:, :3] = x.astype(np.float32)
    xyzq_h[:, 3] = np.asarray(s.charge, np.float32)
    xyzq = torch.from_numpy(xyzq_h).cuda()
    stride = n + 37                      # a stride longer than the atom count
    for call in range(2):                # two calls in a row reuse the static area
        grad = torch.zeros(3 * stride, dtype=torch.int64, device="cuda")
        energy = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = _static_call(torch, xyzq.data_ptr(), n, s.box, nfft, order, 0.34,
                          grad.data_ptr(), stride, energy.data_ptr(), precise)
        assert st == 0, lib().apo_last_error()
        torch.cuda.synchronize()
        if call == 1:
            # the first call may load the kernels' code onto the device; the
            # second allocates nothing: the device's free memory is unchanged
            assert torch.cuda.mem_get_info()[0] == free_before
        G = grad.view(3, stride)[:, :n].t().cpu().numpy().astype(np.float64) / FORCE_SCALE
        rel = np.sqrt(((G - G_ref) ** 2).sum() / (G_ref ** 2).sum())
        assert rel < FORCE_RTOL, (call, rel)
        assert float(energy.item()) == pytest.approx(ewks_ref, rel=ENERGY_RTOL), call
        assert not grad.view(3, stride)[:, n:].any()   # nothing written past the atoms
    # and both against the FP64 reciprocal sum
    Eo, Go = oracle_for(s, settings).evaluate(pos=x, parts=("recip",))
    assert np.sqrt(((G - Go) ** 2).sum() / (Go ** 2).sum()) < FORCE_RTOL
    assert float(energy.item()) == pytest.approx(Eo["ewks"], rel=1e-5)


def test_static_reciprocal_rejects_oversize_and_bad_arguments():
    torch = pytest.importorskip("torch")
    xyzq = torch.zeros((8, 4), dtype=torch.float32, device="cuda")
    grad = torch.zeros(3 * 8, dtype=torch.int64, device="cuda")
    # 96^3 needs more than the 8 MiB static area: refused before any launch
    st = _static_call(torch, xyzq.data_ptr(), 8, (30.0, 30.0, 30.0), (96, 96, 96), 4, 0.34,
                      grad.data_ptr(), 8, None, False)
    assert st == 1  # APO_STATUS_INVALID_ARGUMENT
    msg = lib().apo_last_error()
    msg = msg.decode() if isinstance(msg, bytes) else str(msg)
    assert "static area" in msg
    st = _static_call(torch, xyzq.data_ptr(), 8, (30.0, 30.0, 30.0), (24, 24, 25), 4, 0.34,
                      grad.data_ptr(), 8, None, False)
    assert st == 1
    st = _static_call(torch, xyzq.data_ptr(), 8, (30.0, 30.0, 30.0), (24, 24, 24), 5, 0.34,
                      grad.data_ptr(), 8, None, False)
    assert st == 1
    # a grid axis shorter than the spline order would wrap a spline twice
    st = _static_call(torch, xyzq.data_ptr(), 8, (30.0, 30.0, 30.0), (4, 4, 4), 6, 0.34,
                      grad.data_ptr(), 8, None, False)
    assert st == 1
