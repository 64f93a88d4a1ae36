"""Failure detection on the GPU without a GPU fault: bad inputs and solver
limits come back as status codes, and the context stays usable."""
import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import channel_case, random_fields, to_device

pytestmark = pytest.mark.gpu


def test_nan_in_uploaded_field_is_reported():
    g, bc = channel_case(16, 8, 8)
    f = random_fields(g, 1, scale=0.1)
    f.us[3, 4, 5] = np.nan
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8))
        st = s.pressure_projection(1e-3, check=False)
        assert st.rc == M.MDX_ERR_NONFINITE
        # the context is still usable
        f2 = random_fields(g, 2, scale=0.1)
        s.set("us", f2.us)
        st = s.pressure_projection(1e-3, check=False)
        assert st.rc in (M.MDX_OK, M.MDX_NOT_CONVERGED)


def test_not_converged_status():
    g, bc = channel_case(16, 8, 8)
    f = random_fields(g, 3, scale=0.1)
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-14, max_iter=1, check_every=1))
        st = s.pressure_projection(1e-3, check=False)
        assert st.rc == M.MDX_NOT_CONVERGED and st.iterations == 1


def test_odd_sizes_rejected_for_redblack():
    g, bc = channel_case(15, 8, 8)
    f = random_fields(g, 3)
    with to_device(M, g, bc, f) as s:
        with pytest.raises(M.MdxError) as e:
            s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK))
        assert e.value.code == M.MDX_ERR_ARG


def test_call_order_errors():
    g = M.make_grid(8, 8, 8)
    with M.Solver(g, M.channel_bc()) as s:
        with pytest.raises(M.MdxError) as e:
            s.momentum(1e-3, 0.0, 1e-3)
        assert e.value.code == M.MDX_ERR_STATE
        s.enter_field_data()
        with pytest.raises(M.MdxError) as e:
            s.pressure_projection(1e-3)
        assert e.value.code == M.MDX_ERR_STATE
