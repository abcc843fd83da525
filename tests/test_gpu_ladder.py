"""A DF-JK SCF whose J builds follow the precision ladder on the device:
mixed (FP32-stored B) while the density moves, FP64 after it settles, and an
FP64 exit -- the converged energy equals the all-FP64 DF-RHF energy."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def scf_with_ladder(d, handle, ladder, nocc, max_iter=100, e_tol=1e-12, d_tol=1e-10):
    """The DIIS loop of solve_rhf (ferric-scf/src/rhf.rs:2478-2517) with the
    ladder's begin_build / veto_mixed_exit (jk_ladder.rs:346-430)."""
    from ferric_b200.ladder import REDO_IN_F64
    S, H, enuc = d["s"], d["h_core"], float(d["e_nuc"])
    n = S.shape[0]
    s, u = np.linalg.eigh(S)
    X = u / np.sqrt(s)
    _, c = np.linalg.eigh(X.T @ H @ X)
    C = X @ c
    D = 2.0 * C[:, :nocc] @ C[:, :nocc].T
    focks, errs = [], []
    e_old, d_old = None, None
    builds = {"mixed": 0, "f64": 0}
    E = None
    for _ in range(max_iter):
        mixed = ladder.begin_build([D])
        handle.set_precision("mixed" if mixed else "f64")
        builds["mixed" if mixed else "f64"] += 1
        J = handle.j(D)
        handle.set_precision("f64")          # K on the FP64 path
        Co = C[:, :nocc]
        K = 2.0 * handle.k_from_occ(Co)
        if mixed:
            ladder.note_mixed_build(dfj=True)
        F = H + J - 0.5 * K
        E = 0.5 * np.sum(D * (H + F)) + enuc
        conv = None
        if e_old is not None and abs(E - e_old) < e_tol and d_old is not None and \
                np.abs(D - d_old).max() < d_tol:
            conv = E
        ex = ladder.veto_mixed_exit(conv)
        if ex == REDO_IN_F64:
            focks, errs = [], []                # DIIS history holds mixed Fock matrices
            e_old, d_old = None, None           # invalidate the deltas
            continue                            # rebuild in FP64 at the same density
        if ex is not None:
            return ex, builds
        err = X.T @ (F @ D @ S - S @ D @ F) @ X
        focks.append(F)
        errs.append(err)
        if len(focks) > 8:
            focks.pop(0)
            errs.pop(0)
        m = len(focks)
        B = -np.ones((m + 1, m + 1))
        B[m, m] = 0.0
        for a in range(m):
            for b in range(m):
                B[a, b] = np.sum(errs[a] * errs[b])
        rhs = np.zeros(m + 1)
        rhs[m] = -1.0
        coef = np.linalg.lstsq(B, rhs, rcond=None)[0][:m]
        Fd = sum(cf * f for cf, f in zip(coef, focks))
        _, c = np.linalg.eigh(X.T @ Fd @ X)
        C = X @ c
        e_old, d_old = E, D
        D = 2.0 * C[:, :nocc] @ C[:, :nocc].T
    raise AssertionError("SCF did not converge")


def test_dfjk_scf_under_the_ladder_exits_in_fp64(fc):
    from ferric_b200.dfjk import DfJK
    from ferric_b200.ladder import JkLadder
    d = dict(np.load(os.path.join(GOLDEN, "h2o_ccpvdz.npz")))
    handle = DfJK(d["b_jk"], layout="square", precision="mixed")
    ladder = JkLadder()
    e, builds = scf_with_ladder(d, handle, ladder, int(d["nocc"]))
    assert builds["mixed"] >= 2 and builds["f64"] >= 2
    assert ladder.latched_f64
    assert abs(e - d["oracle_e_dfrhf"]) < 1e-10
    handle.close()
