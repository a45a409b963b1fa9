"""Batched solves (hecmw33_gpu_batch_*): every system of the batch against the
oracle's own hecmw_solve of that system alone, with the drop-in's parity bars
(iterations within +-2, solution within 1e-8 relative, true residual at or below the
tolerance), under every launch schedule the autotuner can pick (single CTAs,
cluster teams of 2 / 4 / 8 CTAs, 4 / 8 / 16 lanes per sweep row), plus the per-system
codes: 2002 (zero load), 2001 (zero diagonal, not solved), 3001 (MAXIT)."""
import numpy as np
import pytest

from frontistr_b200.batch import BatchSolver, stack_systems
from frontistr_b200.mesh import random_box_batch
from oracle_ctypes import Oracle

pytestmark = pytest.mark.gpu


def flags(m, precond=1, maxit=20000, tol=1e-8):
    ia, ra = m.Iarray.copy(), m.Rarray.copy()
    ia[0] = maxit
    ia[2] = precond
    ra[0] = tol
    return ia, ra


def oracle_solutions(systems, precond=1):
    out = []
    for m in systems:
        ia, _ = flags(m, precond)
        out.append(Oracle(m.copy()).solve(Iarray=ia))
    return out


@pytest.fixture(scope="module")
def batch12():
    systems = random_box_batch(12, edge_range=(2, 9), seed=21)
    big, sys_ptr = stack_systems(systems)
    return systems, big, sys_ptr, oracle_solutions(systems)


def check_against_oracle(systems, sys_ptr, X, rec, refs):
    for s, m in enumerate(systems):
        a, e = 3 * sys_ptr[s], 3 * sys_ptr[s + 1]
        ref = refs[s]
        assert rec["errors"][s] == 0, (s, rec["errors"])
        assert abs(int(rec["iter"][s]) - ref["iter"]) <= 2, (s, rec["iter"][s], ref["iter"])
        err = np.linalg.norm(X[a:e] - ref["X"]) / np.linalg.norm(ref["X"])
        assert err <= 1e-8, (s, err)
        tr = Oracle(m).rel_resid(X[a:e], m.B)
        assert tr <= 1e-8
        assert abs(rec["true_resid"][s] - tr) <= 1e-4 * tr  # cancellation in b - A x near 1e-8


@pytest.mark.parametrize("schedule", ["8,1,0", "8,2,0.3", "8,4,0.5", "8,8,1.0", "4,4,0.25", "16,2,0.25"])
def test_batch_matches_oracle_every_schedule(batch12, schedule, monkeypatch):
    systems, big, sys_ptr, refs = batch12
    monkeypatch.setenv("HECMW33_BATCH_SCHEDULE", schedule)
    ia, ra = flags(big)
    X = np.zeros(3 * big.N)
    with BatchSolver() as bs:
        bs.set_matrix(big, sys_ptr, ia, ra)
        rec = bs.solve(big.B, X, ia, ra)
        info = bs.info()
    lanes, cluster, frac = schedule.split(",")
    assert info["lanes"] == int(lanes) and info["cluster"] == int(cluster)
    if int(cluster) > 1:
        assert info["big"] == int(round(float(frac) * 12))
    assert rec["error"] == 0 and ia[80] == 1 and ia[81] == 0
    check_against_oracle(systems, sys_ptr, X, rec, refs)


def test_batch_repeat_and_values_update(batch12, monkeypatch):
    """Second solve on the same handle (graph reused) and a values-only update.  With
    single-CTA teams every system's arithmetic is fixed, so repeats are bitwise equal
    (with cluster teams a system's team size may change between solves when the work
    estimates do)."""
    systems, big, sys_ptr, refs = batch12
    monkeypatch.setenv("HECMW33_BATCH_SCHEDULE", "8,1,0")
    ia, ra = flags(big)
    with BatchSolver() as bs:
        bs.set_matrix(big, sys_ptr, ia, ra)
        X1 = np.zeros(3 * big.N)
        bs.solve(big.B, X1, ia.copy(), ra)
        X2 = np.zeros(3 * big.N)
        rec = bs.solve(big.B, X2, ia.copy(), ra)
        assert np.array_equal(X1, X2)  # deterministic reductions
        check_against_oracle(systems, sys_ptr, X2, rec, refs)
        # scale every matrix by 2: same structure, new values -> x halves
        scaled = big.copy()
        scaled.D *= 2.0
        scaled.AL *= 2.0
        scaled.AU *= 2.0
        ia2 = ia.copy()
        ia2[97] = 0
        bs.set_matrix(scaled, sys_ptr, ia2, ra)
        X3 = np.zeros(3 * big.N)
        rec3 = bs.solve(big.B, X3, ia.copy(), ra)
        assert rec3["error"] == 0
        assert np.linalg.norm(2.0 * X3 - X2) <= 1e-7 * np.linalg.norm(X2)


def test_batch_codes_zero_rhs_zero_diag_maxit(monkeypatch):
    monkeypatch.setenv("HECMW33_BATCH_SCHEDULE", "8,2,0.5")
    systems = random_box_batch(5, edge_range=(2, 5), seed=4)
    systems[1].B[:] = 0.0                 # zero load case
    systems[3].D[0] = 0.0                 # zero diagonal entry (node 0 of system 3)
    big, sys_ptr = stack_systems(systems)
    ia, ra = flags(big)
    X = np.ones(3 * big.N)
    with BatchSolver() as bs:
        bs.set_matrix(big, sys_ptr, ia, ra)
        rec = bs.solve(big.B, X, ia, ra)
        assert rec["errors"][1] == 2002
        assert np.all(X[3 * sys_ptr[1]:3 * sys_ptr[2]] == 0.0)
        assert rec["errors"][3] == 2001
        assert np.all(X[3 * sys_ptr[3]:3 * sys_ptr[4]] == 1.0)  # not solved, X untouched
        for s in (0, 2, 4):
            assert rec["errors"][s] == 0
            a, e = 3 * sys_ptr[s], 3 * sys_ptr[s + 1]
            assert Oracle(systems[s]).rel_resid(X[a:e], systems[s].B) <= 1e-8
        assert rec["error"] == 2001 and ia[80] == 0
        # MAXIT for every system
        ia3, ra3 = flags(big, maxit=3)
        X = np.zeros(3 * big.N)
        rec = bs.solve(big.B, X, ia3, ra3)
        assert [int(v) for v in rec["errors"]] == [3001, 2002, 3001, 2001, 3001]
        assert [int(rec["iter"][s]) for s in (0, 2, 4)] == [4, 4, 4]


def test_batch_diag_preconditioner(monkeypatch):
    monkeypatch.setenv("HECMW33_BATCH_SCHEDULE", "8,4,0.34")
    systems = random_box_batch(6, edge_range=(2, 6), seed=8)
    refs = oracle_solutions(systems, precond=3)
    big, sys_ptr = stack_systems(systems)
    ia, ra = flags(big, precond=3)
    X = np.zeros(3 * big.N)
    with BatchSolver() as bs:
        bs.set_matrix(big, sys_ptr, ia, ra)
        rec = bs.solve(big.B, X, ia, ra)
    check_against_oracle(systems, sys_ptr, X, rec, refs)


def test_batch_autotune_and_cache(batch12, tmp_path, monkeypatch):
    systems, big, sys_ptr, refs = batch12
    cache = tmp_path / "tune.jsonl"
    monkeypatch.setenv("HECMW33_AUTOTUNE_CACHE", str(cache))
    monkeypatch.delenv("HECMW33_BATCH_SCHEDULE", raising=False)
    ia, ra = flags(big)
    X0 = np.zeros(3 * big.N)
    with BatchSolver() as bs:
        bs.set_matrix(big, sys_ptr, ia, ra)
        info = bs.autotune(big.B, X0, ia, ra)
        assert info["tuned"] == 1
        assert np.all(X0 == 0.0)  # the autotuner leaves the caller's X alone
    lines = cache.read_text().strip().splitlines()
    assert len(lines) == 1 and '"lanes": %d' % info["lanes"] in lines[0]
    with BatchSolver() as bs:  # a new handle picks the schedule up from the cache
        bs.set_matrix(big, sys_ptr, ia, ra)
        X = np.zeros(3 * big.N)
        rec = bs.solve(big.B, X, ia, ra)
        info2 = bs.info()
    assert info2["tuned"] == 1 and (info2["lanes"], info2["cluster"]) == (info["lanes"], info["cluster"])
    check_against_oracle(systems, sys_ptr, X, rec, refs)
