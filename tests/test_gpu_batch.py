"""Batched evaluation: persistent fused launches over many molecules (the factored density matrices
on one, the others on another), the staged path for the large ones, Hockney solves with tuned
padding, all captured in one CUDA graph.  Each molecule's result must equal its single-molecule
evaluation through the facade."""
import ctypes as C

import numpy as np
import pytest

import qmtools
from qmtools import _native as N
from qmtools import synthetic as syn
from qmtools.autotune import PATH_FACTORED, PATH_FUSED, PATH_STAGED, Tuner, fft_candidates
from qmtools.batch import BatchEvaluator

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mols(basis):
    # 3, 9, 20, 33 (N > 320: staged) and 12 atoms; grids of the batch workload (bbox + 3 bohr),
    # made smaller with a coarser step so the test stays short
    out = []
    for i, n in enumerate((3, 9, 20, 33, 12)):
        sm = syn.extent_molecule(n, 900 + i, step=0.45)
        out.append((sm, sm.molecule(basis, qmtools.Molecule), sm.grid(qmtools.Grid)))
    return out


def _single(mol, g, m_lengths, path):
    """One molecule through the facade, on the density path the batch's tuner chose for it."""
    import torch
    N.call("qmt_set_density_path", int(path))
    try:
        q = qmtools.QMTools.Compute_density(g, mol, precision="fp16x3", copyBack=False)
    finally:
        N.call("qmt_set_density_path", 0)
    nx, ny, nz, h, ox, oy, oz = g._geom()
    v = torch.empty(nx * ny * nz, device="cuda")
    mx, my, mz = m_lengths
    N.call("qmt_fft_poisson_padded", mol.handle, nx, ny, nz, h, ox, oy, oz, 0.2, 6.0, mx, my, mz,
           C.c_void_p(q.field(0).data_ptr()), C.c_void_p(v.data_ptr()), N.stream_handle())
    return q.field(0).cpu().numpy(), v.cpu().numpy().reshape(nx, ny, nz)


@pytest.mark.parametrize("measure", [False, True], ids=["default_paths", "tuned_paths"])
def test_batch_equals_single_molecule_evaluations(mols, tmp_path, measure):
    """Every molecule takes its factored density matrix (the synthetic matrices have rank n_occ):
    the four small ones on one persistent fused launch, the large one (N > 320) on the staged path;
    with measured or default tuner choices alike."""
    tuner = Tuner(path=tmp_path / "tune.json", measure=measure)
    ev = BatchEvaluator([m for _, m, _ in mols], [g for _, _, g in mols], tuner=tuner)
    try:
        assert all(p == PATH_FACTORED for p in ev.paths)
        assert ev.fused_count == 4                      # the fifth has N > 320: staged
        assert ev.factored_count == 5
        first = None
        for rep in range(2):                            # two graph replays
            ev.run()
            ev.synchronize()
            grids = [(ev.density(i), ev.potential(i)) for i in range(len(mols))]
            if first is None:
                first = grids
            for i, (sm, mol, g) in enumerate(mols):
                q, v = grids[i]
                # replays repeat themselves exactly
                assert np.array_equal(q, first[i][0]) and np.array_equal(v, first[i][1]), (rep, i)
                q1, v1 = _single(mol, g, ev.fft_lengths[i], ev.paths[i])
                if ev.paths[i] == PATH_FACTORED and ev.fused_count > 1 and i != 3:
                    # the factored launch over several molecules is another compilation of the
                    # same arithmetic (the kernel template for many molecules): equal to rounding
                    assert np.abs(q - q1).max() <= 4e-7 * np.abs(q1).max(), (rep, i)
                    assert np.linalg.norm(v - v1) <= 1e-6 * np.linalg.norm(v1), (rep, i)
                else:
                    assert np.array_equal(q, q1), (rep, i)
                    assert np.array_equal(v, v1), (rep, i)
        sums = ev.sums()
        assert np.all(np.isfinite(sums)) and np.all(sums > 0)
        if measure:
            assert (tmp_path / "tune.json").exists() and tuner.measured > 0
    finally:
        ev.close()


def test_batch_graph_follows_new_density_matrices(mols, tmp_path):
    """With refresh the captured graph re-derives the split density matrices from new uploads (and
    keeps the unfactored matrices: a factor is built on the host)."""
    sel = [mols[0], mols[2]]
    ev = BatchEvaluator([m for _, m, _ in sel], [g for _, _, g in sel], tuner=Tuner(path=tmp_path / "t.json"),
                        refresh=True)
    try:
        assert ev.factored_count == 0 and PATH_FACTORED not in ev.paths
        rng = np.random.default_rng(3)
        saved = [np.array(m.dm) for _, m, _ in sel]
        for (_, m, _), dm in zip(sel, saved):
            d2 = dm * (1.0 + 0.05 * rng.standard_normal(dm.shape))
            m.set_dm(0.5 * (d2 + d2.T))
        import torch
        torch.cuda.synchronize()
        ev.run()
        ev.synchronize()
        for i, (_, m, g) in enumerate(sel):
            q1, v1 = _single(m, g, ev.fft_lengths[i], ev.paths[i])
            assert np.array_equal(ev.density(i), q1)
            assert np.array_equal(ev.potential(i), v1)
        for (_, m, _), dm in zip(sel, saved):
            m.set_dm(dm)
    finally:
        ev.close()


def test_tuner_cache_is_reused(mols, tmp_path):
    path = tmp_path / "tune.json"
    t1 = Tuner(path=path)
    _, mol, g = mols[1]
    p1 = t1.density_path(mol, int(g.npts), "fp16x3")
    m1 = t1.fft_length(40, mol)
    assert p1 in (PATH_FUSED, PATH_STAGED) and m1 in fft_candidates(40)
    t2 = Tuner(path=path)
    assert t2.density_path(mol, int(g.npts), "fp16x3") == p1 and t2.fft_length(40, mol) == m1
    assert t2.measured == 0
