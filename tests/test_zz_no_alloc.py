"""GPU tests of gpx_cap_solve_small_static, the entry point that computes a
small problem's Maxwell matrix in the library's fixed static device scratch
instead of allocating.  It is compared, through the C ABI, with gpx_cap_solve
on its all-pairs path (the same dense system, solved there by GMRES to a
1e-12 relative residual, here by LU), on two calls in a row; sizes beyond
its limits, host pointers and bad conductor indices give an error status.

Bar: 1e-9 relative to the largest entry, as for the all-pairs path against the
oracle's LU.  The file is named so that it is collected last."""
import numpy as np
import pytest

from gpurify_b200 import _lib, layouts
from tests.helpers import rel_max

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = _lib.Context(0)
    yield c
    c.close()


def _plate(x0, y0, z, w, h, nx, ny, cond):
    """nx x ny quads of a horizontal w x h plate at height z (metres)."""
    xs = np.linspace(x0, x0 + w, nx + 1)
    ys = np.linspace(y0, y0 + h, ny + 1)
    v = []
    for i in range(nx):
        for j in range(ny):
            v.append([xs[i], ys[j], z, xs[i + 1], ys[j], z, xs[i + 1], ys[j + 1], z, xs[i], ys[j + 1], z])
    return np.array(v), np.full(len(v), cond, np.int32)


def _three_conductors():
    a, ca = _plate(0.0, 0.0, 1.0e-6, 4.0e-6, 4.0e-6, 14, 14, 0)
    b, cb = _plate(1.0e-6, 0.5e-6, 1.6e-6, 3.0e-6, 3.0e-6, 14, 14, 1)
    g, cg = _plate(-2.0e-6, -2.0e-6, 0.0, 8.0e-6, 8.0e-6, 10, 10, 2)
    return np.vstack([a, b, g]), np.concatenate([ca, cb, cg]), 3


def _max_size():
    a, ca = _plate(0.0, 0.0, 0.0, 2.0e-6, 2.0e-6, 16, 16, 0)
    b, cb = _plate(0.0, 0.0, 0.3e-6, 2.0e-6, 2.0e-6, 16, 16, 1)
    return np.vstack([a, b]), np.concatenate([ca, cb]), 2


def _short_wires():
    lay = layouts.two_wires(length_nm=3000)
    p = _lib.bridge_panelize(lay.store.arrays(), lay.deck.layer_table(), 1.0, lay.net_of_poly)
    return p["verts"], p["cond"], len(p["nets"]) + 1


CASES = {"three_conductors_492": _three_conductors, "max_size_512": _max_size, "bridge_two_wires": _short_wires}


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


@pytest.mark.parametrize("case", sorted(CASES))
def test_matches_cap_solve_on_two_calls(ctx, case):
    verts, cond, ncond = CASES[case]()
    assert len(verts) <= 512
    ref, rep = ctx.cap_solve(verts, cond, ncond, dense_below=1024)
    assert rep["dense"] == 1 and rep["converged"] == 1
    dv, dc = _dev(verts.astype(np.float64)), _dev(cond.astype(np.int32))
    out = torch.full((ncond * ncond,), float("nan"), dtype=torch.float64, device="cuda:0")
    results = []
    for _ in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        ctx.cap_solve_small_static(len(verts), dv.data_ptr(), dc.data_ptr(), ncond, out.data_ptr())
        C = out.cpu().numpy().reshape(ncond, ncond)
        assert np.isfinite(C).all()
        assert rel_max(C, ref) < 1e-9, (case, rel_max(C, ref))
        results.append(C)
    assert rel_max(results[1], results[0]) < 1e-12


def test_second_call_takes_no_device_memory(ctx):
    """After a first call on the device (the one-time set-up, which loads every
    kernel of the entry point), a call that also runs the LU's trailing update
    (above 32 panels) leaves the device's free memory unchanged."""
    verts, cond, ncond = _short_wires()
    assert len(verts) > 32
    dv, dc = _dev(verts.astype(np.float64)), _dev(cond.astype(np.int32))
    out = torch.zeros(ncond * ncond, dtype=torch.float64, device="cuda:0")
    small_v, small_c = dv[:8].contiguous(), torch.zeros(8, dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    # warm-up on 8 panels: no trailing update runs in this call
    ctx.cap_solve_small_static(8, small_v.data_ptr(), small_c.data_ptr(), 1, out.data_ptr())
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    ctx.cap_solve_small_static(len(verts), dv.data_ptr(), dc.data_ptr(), ncond, out.data_ptr())
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
    assert np.isfinite(out.cpu().numpy()).all()


def test_rejects_inputs_beyond_its_limits(ctx):
    verts, cond, ncond = _max_size()
    dv, dc = _dev(verts), _dev(cond)
    out = torch.zeros(64 * 64, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    with pytest.raises(_lib.GpxError, match=r"n_panels = 513 .*\[1, 512\]"):
        ctx.cap_solve_small_static(513, dv.data_ptr(), dc.data_ptr(), ncond, out.data_ptr())
    with pytest.raises(_lib.GpxError, match=r"n_conductors = 65 .*\[1, 64\]"):
        ctx.cap_solve_small_static(len(verts), dv.data_ptr(), dc.data_ptr(), 65, out.data_ptr())
    host = np.ascontiguousarray(verts)
    with pytest.raises(_lib.GpxError, match="device"):
        ctx.cap_solve_small_static(len(verts), host.ctypes.data, dc.data_ptr(), ncond, out.data_ptr())
    bad = _dev(np.where(np.arange(len(cond)) == 7, 5, cond).astype(np.int32))
    with pytest.raises(_lib.GpxError, match="conductor index"):
        ctx.cap_solve_small_static(len(verts), dv.data_ptr(), bad.data_ptr(), ncond, out.data_ptr())
    # a rejected call leaves the entry point usable
    ctx.cap_solve_small_static(len(verts), dv.data_ptr(), dc.data_ptr(), ncond, out.data_ptr())
    assert np.isfinite(out[: ncond * ncond].cpu().numpy()).all()
