"""Continuous batching: results are the same alone and in the mix; admission by HBM footprint."""
import numpy as np
import pytest

import qmtools
from qmtools import serving
from qmtools import synthetic as syn
from oracle import density as od
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _requests(basis, n=6, seed=11):
    reqs = []
    rng = np.random.default_rng(seed)
    for i in range(n):
        sm = syn.extent_molecule(int(rng.integers(3, 14)), seed * 100 + i, step=0.4)
        mol = sm.molecule(basis, qmtools.Molecule)
        reqs.append(serving.Request(mol, sm.grid(qmtools.Grid), arrival=0.002 * i, rid=i))
    return reqs


def test_alone_equals_mixed(basis):
    alone = _requests(basis)
    eng = serving.Engine(slots=1)
    eng.run(alone, realtime=False)
    eng.close()
    mixed = _requests(basis)
    eng = serving.Engine(slots=4)
    eng.run(mixed, realtime=True)
    eng.close()
    for a, m in zip(alone, mixed):
        assert a.rid == m.rid
        assert np.array_equal(a.density, m.density)
        assert np.array_equal(a.potential, m.potential)
        assert m.latency is not None and m.latency > 0
    stats = serving.latency_stats(mixed)
    assert stats["n"] == len(mixed) and stats["p99_ms"] >= stats["p50_ms"]


def test_served_density_matches_oracle(basis):
    reqs = _requests(basis, n=2, seed=5)
    eng = serving.Engine(slots=2)
    eng.run(reqs, realtime=False)
    eng.close()
    for r in reqs:
        nx, ny, nz, h, ox, oy, oz = r.grid._geom()
        mol = r.molecule
        ref, _, _ = od.compute_density((nx, ny, nz), np.float32(h), (ox, oy, oz), mol.coords, mol.types, mol.ALMOs,
                                       mol.basisset.alphas, mol.basisset.coeffs, mol.dm)
        assert rel_l2(r.density, ref) < 1e-6
        assert abs(float(r.density.sum(dtype=np.float64)) - float(mol.qtot)) < 1e-3


def test_budget_serialises_admission(basis):
    reqs = _requests(basis, n=3, seed=7)
    need = max(serving.footprint(r) for r in reqs)
    eng = serving.Engine(slots=3, hbm_budget=need)     # room for one request at a time
    eng.run(reqs, realtime=False)
    eng.close()
    order = sorted(reqs, key=lambda r: r.t_admit)
    for prev, nxt in zip(order, order[1:]):
        assert nxt.t_admit >= prev.t_done - 1e-6
    with pytest.raises(qmtools._native.QMToolsError):
        serving.Engine(slots=1, hbm_budget=need // 4).run(_requests(basis, n=1), realtime=False)
