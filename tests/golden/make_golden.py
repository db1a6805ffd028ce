"""Regenerates tests/golden/golden.npz from the reference-built oracle
(oracle/_ref/libmtlref.so: MTL4's own headers compiled unchanged).

    make -C oracle ref && python tests/golden/make_golden.py

The fixtures pin the oracle restatement and the GPU library on machines
where the MTL4 tree is not available.
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from mtl4_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    out = {}
    # 2D Laplacian (laplacian_setup) 32x32: CSR, SpMV, CG runs
    A = P.laplacian_2d(32)
    x_true, b = P.rhs_from_solution(A, 0)
    R = O.RefMatrix(A)
    rp, ci, v = O.ref_laplacian(32, 32)
    out["lap32_rp"], out["lap32_ci"], out["lap32_val"] = rp, ci, v
    xs = np.random.default_rng(11).standard_normal(A.n_rows)
    out["lap32_x"] = xs
    out["lap32_spmv"] = R.spmv(xs)
    out["lap32_spmv_f32"] = R.spmv(xs.astype(np.float32))
    out["lap32_b"] = b
    for solver, pc in [("cg", "diagonal"), ("cg", "identity"), ("cg", "ic_0"), ("bicgstab", "ilu_0"),
                       ("bicgstab", "diagonal"), ("bicgstab", "identity"), ("bicgstab", "ic_0")]:
        r = R.solve(b, solver, pc, max_iter=2000, rtol=1e-8)
        out[f"lap32_{solver}_{pc}_iters"] = np.array(r["iterations"])
        out[f"lap32_{solver}_{pc}_x"] = r["x"]
        out[f"lap32_{solver}_{pc}_relres"] = np.array(r["relresid"])
    # 3D convection-diffusion 8^3: factors and applies in all precisions
    C3 = P.convdiff_3d(8)
    out["cd8_rp"], out["cd8_ci"], out["cd8_val"] = C3.row_ptr, C3.col, C3.val
    R3 = O.RefMatrix(C3)
    xc = np.random.default_rng(12).standard_normal(C3.n_rows)
    out["cd8_x"] = xc
    for kind in ["ilu_0", "ic_0"]:
        (Lr, Lc, Lv), (Ur, Uc, Uv) = R3.factors(kind)
        out[f"cd8_{kind}_L_rp"], out[f"cd8_{kind}_L_ci"], out[f"cd8_{kind}_L_val"] = Lr, Lc, Lv
        out[f"cd8_{kind}_U_rp"], out[f"cd8_{kind}_U_ci"], out[f"cd8_{kind}_U_val"] = Ur, Uc, Uv
    for kind in ["diagonal", "ilu_0", "ic_0"]:
        out[f"cd8_{kind}_apply_f64"] = R3.pc_apply(kind, xc)
        out[f"cd8_{kind}_apply_f64s32"] = R3.pc_apply(kind, xc, storage_f32=True)
        out[f"cd8_{kind}_apply_f32"] = R3.pc_apply(kind, xc.astype(np.float32))
    _, b3 = P.rhs_from_solution(C3, 1)
    out["cd8_b"] = b3
    r = R3.solve(b3, "bicgstab", "ilu_0", max_iter=500, rtol=1e-8)
    out["cd8_bicgstab_ilu_0_iters"] = np.array(r["iterations"])
    # irregular power-law CSR (small)
    Q = P.powerlaw_csr(5000, seed=2)
    out["pl_rp"], out["pl_ci"], out["pl_val"] = Q.row_ptr, Q.col, Q.val
    RQ = O.RefMatrix(Q)
    xq = np.random.default_rng(13).standard_normal(Q.n_rows)
    out["pl_x"] = xq
    out["pl_spmv"] = RQ.spmv(xq)
    out["pl_spmv_f32"] = RQ.spmv(xq.astype(np.float32))
    # itl::cyclic_iteration output of the reference's loops (per-cycle residual
    # lines and the summary the solver's return prints)
    for solver, pc, cycle, multi in [("cg", "diagonal", 10, 0), ("bicgstab", "ilu_0", 1, 0),
                                     ("bicgstab", "identity", 5, 1)]:
        err, text = R.solve_cyclic(b, solver, pc, max_iter=2000, rtol=1e-8, cycle=cycle, multi_print=bool(multi))
        out[f"lap32_{solver}_{pc}_cyclic{cycle}_{multi}"] = np.array(text)
    # ELL and sparse_banded forms (ell_matrix / sparse_banded = compressed2D)
    # and their products on the 8^3 convection-diffusion operator and on a
    # rectangular banded matrix with bands that end inside it
    st, sl, mi, da = R3.ell()
    out["cd8_ell_stride"], out["cd8_ell_slots"] = np.array(st), np.array(sl)
    out["cd8_ell_minor"], out["cd8_ell_data"] = mi, da
    out["cd8_ell_y"] = R3.ell_spmv(xc)
    bands, bd = R3.banded()
    out["cd8_band_bands"], out["cd8_band_data"] = bands, bd
    out["cd8_band_y"] = R3.banded_spmv(xc)
    rb = np.random.default_rng(15)
    offs = [-37, -5, -2, 0, 3, 19, 60]
    nr, nc = 203, 231
    rows, cols = [], []
    for o in offs:
        r = np.arange(max(0, -o), min(nr, nc - o))
        rows.append(r)
        cols.append(r + o)
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    Bm = P._from_coo(nr, rows, cols, rb.standard_normal(rows.size))
    Bm = P.CSR(nr, nc, Bm.row_ptr, Bm.col, Bm.val)
    RB = O.RefMatrix(Bm)
    out["rb_rp"], out["rb_ci"], out["rb_val"] = Bm.row_ptr, Bm.col, Bm.val
    out["rb_x"] = rb.standard_normal(nc)
    out["rb_y0"] = rb.standard_normal(nr)
    bands, bd = RB.banded()
    out["rb_bands"], out["rb_data"] = bands, bd
    for a in (0, 1, 2):
        out[f"rb_band_y{a}"] = RB.banded_spmv(out["rb_x"], a, out["rb_y0"])
        out[f"rb_ell_y{a}"] = RB.ell_spmv(out["rb_x"], a, out["rb_y0"])
    # mtl::dot and mtl::two_norm (four strided partial sums) on general values
    out["dot_x"] = xq[:1001]
    out["dot_y"] = np.random.default_rng(14).standard_normal(1001)
    out["dot_xy"] = np.array(O.ref_lib().mtlref_dot(1001, O._p(out["dot_x"]), O._p(out["dot_y"])))
    out["norm_x"] = np.array(O.ref_lib().mtlref_two_norm(1001, O._p(out["dot_x"])))
    # full-size solves: iteration counts, relative residuals and the SHA-256 of
    # the solution's bytes (the reference's x itself is too large to keep)
    for tag, (A_, b_), solver, pc in [("c1", P.config1()[:2], "cg", "diagonal"),
                                      ("c2", P.config2_solve(128)[:2], "bicgstab", "ilu_0")]:
        r = O.RefMatrix(A_).solve(b_, solver, pc, max_iter=2000, rtol=1e-8)
        out[f"{tag}_iters"] = np.array(r["iterations"])
        out[f"{tag}_relres"] = np.array(r["relresid"])
        out[f"{tag}_x_sha256"] = np.array(hashlib.sha256(np.ascontiguousarray(r["x"]).tobytes()).hexdigest())
    np.savez_compressed(Path(__file__).with_name("golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
