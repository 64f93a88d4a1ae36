"""IBM coefficients generated on the device (set_ibm_coeff, ibm.f90:133-187)
against the host routine, and a step with device-generated coefficients
against one with host-generated ones."""
import math

import numpy as np
import pytest
import torch

import mobydiff_b200 as M
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

COMPONENTS = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]


def _grid(nx, ny, nz, ly=2.25):
    return M.make_grid(nx, ny, nz, 2 * math.pi, ly, math.pi, 3000.0, 1e-3, (2.0 / 3000.0, 0.0, 0.0))


def _device_coeff(g, geom, dd):
    n = (g.nx + 2) * (g.ny + 2) * (g.nz + 2)
    buf = torch.full((n,), -1.0, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    M._check(M.lib().mdx_set_ibm_coeff_device(M.C.byref(g), M.C.byref(geom), buf.data_ptr(), *dd, None))
    torch.cuda.synchronize()
    return buf.cpu().numpy().reshape(g.nz + 2, g.ny + 2, g.nx + 2)


@pytest.mark.parametrize("shape", [(32, 16, 16), (64, 48, 24), (100, 30, 12)])
@pytest.mark.parametrize("kind", ["reference", "wavy"])
def test_device_coefficients_match_host(shape, kind):
    g = _grid(*shape)
    geom = M.ibm_reference(g) if kind == "reference" else M.ibm_wavy(0.05, g.lx / 2, (g.ly - 2.0) / 2.0)
    host = M.set_ibm_coeff(g, geom)
    for dd, h in zip(COMPONENTS, host):
        dev = _device_coeff(g, geom, dd)
        h = h.reshape(dev.shape)
        solid = h >= 1e20
        assert solid.any() and (~solid).any()
        assert np.array_equal(dev >= 1e20, solid), dd
        exact = dev == h
        # the device sin may round differently in the last bit: only a point
        # within one rounding of the wall can move, by a bisection tolerance
        assert exact.mean() >= 0.999, (dd, exact.mean())
        fluid = ~solid
        assert np.max(np.abs(dev[fluid] - h[fluid]) / np.maximum(np.abs(h[fluid]), 1e-300)) <= 1e-6, dd
        # walls depend on x and y only
        assert np.array_equal(dev, np.broadcast_to(dev[:1], dev.shape)), dd


def test_bad_geometry_is_refused():
    g = _grid(32, 16, 16)
    bad = M.ibm_wavy(0.05, 0.0, 0.0)   # wavelength 0
    buf = torch.zeros(34 * 18 * 18, dtype=torch.float64, device="cuda:0")
    assert M.lib().mdx_set_ibm_coeff_device(M.C.byref(g), M.C.byref(bad), buf.data_ptr(), 1, 0, 0, None) != 0
    s = M.Solver(g, M.channel_bc(), 0)
    with s:
        s.enter_field_data()
        with pytest.raises(M.MdxError):
            s.enter_ibm_geometry(bad)


def test_step_with_device_coefficients():
    """The context's mirrors hold the device coefficients, and steps from
    them agree with steps from the host coefficients."""
    g = _grid(64, 32, 32)
    geom = M.ibm_wavy(0.05, g.lx / 2, (g.ly - 2.0) / 2.0)
    y0 = (g.ly - 2.0) / 2.0
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8, check_every=10, max_iter=200000)
    sd, sh = M.Solver(g, M.channel_bc(), 0), M.Solver(g, M.channel_bc(), 0)
    with sd, sh:
        for s in (sd, sh):
            s.enter_field_data()
        sd.enter_ibm_geometry(geom)
        host = M.set_ibm_coeff(g, geom)
        sh.enter_ibm_data(*host)
        same = True
        for name, h in zip(("coef_u", "coef_v", "coef_w"), host):
            dev = sd.get(name)
            same = same and np.array_equal(dev.ravel(), h.ravel())
            assert np.array_equal(dev >= 1e20, h.reshape(dev.shape) >= 1e20), name
        for s in (sd, sh):
            s.init_pressure_solver(opts)
            s.channel_ic(7, 0.1, 0.01, y0, 0.05, g.lx / 2)
        sd.step(3)
        sh.step(3)
        for n in ("un", "vn", "wn", "pn"):
            if same:
                assert np.array_equal(sd.get(n), sh.get(n)), n
            else:
                assert rel_l2(sd.get(n), sh.get(n)) <= 1e-6, n
