"""ELL and sparse_banded forms (the reference's ell_matrix and sparse_banded,
operation/mat_vec_mult.hpp:686-803): the library's host layouts equal the
reference's, the oracle's products are bitwise the reference's (fixtures from
the reference build), and on the GPU the device products are bitwise the
same."""
import numpy as np
import pytest

from conftest import csr_from
from mtl4_b200 import problems as P
from mtl4_b200.mtl import banded_layout, ell_layout
from oracle import oracle as O


def rb_csr(golden):
    A = csr_from(golden, "rb")
    return P.CSR(A.n_rows, golden["rb_x"].size, A.row_ptr, A.col, A.val)


def test_layouts_equal_the_references(golden):
    A = csr_from(golden, "cd8")
    st, sl, mi, da = ell_layout(A)
    assert (st, sl) == (int(golden["cd8_ell_stride"]), int(golden["cd8_ell_slots"]))
    assert np.array_equal(mi, golden["cd8_ell_minor"]) and np.array_equal(da, golden["cd8_ell_data"])
    bands, data = banded_layout(A)
    assert np.array_equal(bands, golden["cd8_band_bands"]) and np.array_equal(data, golden["cd8_band_data"])
    B = rb_csr(golden)
    bands, data = banded_layout(B)
    assert np.array_equal(bands, golden["rb_bands"]) and np.array_equal(data, golden["rb_data"])


def test_oracle_products_bitwise_golden(golden):
    A = csr_from(golden, "cd8")
    x = golden["cd8_x"]
    y = O.port_ell_spmv(A.n_rows, int(golden["cd8_ell_stride"]), int(golden["cd8_ell_slots"]),
                        golden["cd8_ell_minor"], golden["cd8_ell_data"], x)
    assert np.array_equal(y, golden["cd8_ell_y"])
    y = O.port_banded_spmv(A.n_rows, A.n_cols, golden["cd8_band_bands"], golden["cd8_band_data"], x)
    assert np.array_equal(y, golden["cd8_band_y"])
    B = rb_csr(golden)
    st, sl, mi, da = ell_layout(B)
    for a in (0, 1, 2):
        yb = O.port_banded_spmv(B.n_rows, B.n_cols, golden["rb_bands"], golden["rb_data"], golden["rb_x"], a,
                                golden["rb_y0"])
        assert np.array_equal(yb, golden[f"rb_band_y{a}"]), a
        ye = O.port_ell_spmv(B.n_rows, st, sl, mi, da, golden["rb_x"], a, golden["rb_y0"])
        assert np.array_equal(ye, golden[f"rb_ell_y{a}"]), a


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["ell", "banded"])
def test_device_products_bitwise(ctx, golden, fmt):
    from mtl4_b200 import mtl
    cls = mtl.ell_matrix if fmt == "ell" else mtl.sparse_banded
    B = rb_csr(golden)
    Bd = cls.from_csr(B, ctx)
    x = mtl.dense_vector(golden["rb_x"], np.float64, ctx)
    for a, op in ((0, "="), (1, "+="), (2, "-=")):
        y = mtl.dense_vector(golden["rb_y0"], np.float64, ctx)
        mtl.mult(Bd, x, y, op)
        assert np.array_equal(y.numpy(), golden[f"rb_{'ell' if fmt == 'ell' else 'band'}_y{a}"]), op
    # larger operators against the oracle, and FP32
    for A in (P.convdiff_3d(30), P.vardiff_2d(300, sigma=0.7, seed=3)):
        Ad = cls.from_csr(A, ctx)
        xv = np.random.default_rng(2).standard_normal(A.n_cols)
        y = mtl.dense_vector(A.n_rows, np.float64, ctx)
        mtl.mult(Ad, mtl.dense_vector(xv, np.float64, ctx), y)
        if fmt == "ell":
            st, sl, mi, da = ell_layout(A)
            want = O.port_ell_spmv(A.n_rows, st, sl, mi, da, xv)
        else:
            bands, data = banded_layout(A)
            want = O.port_banded_spmv(A.n_rows, A.n_cols, bands, data, xv)
        assert np.array_equal(y.numpy(), want)
        yf = mtl.dense_vector(A.n_rows, np.float32, ctx)
        mtl.mult(Ad, mtl.dense_vector(xv.astype(np.float32), np.float32, ctx), yf)
        scale = np.abs(A.to_scipy()) @ np.abs(xv) + 1e-30
        assert (np.abs(yf.numpy() - want) / scale).max() <= 1e-6
