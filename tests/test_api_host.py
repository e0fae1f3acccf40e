"""Host-side behaviour of the drop-in API (no GPU): parsing, geometry, file formats."""
import pickle
import struct

import numpy as np
import pytest

import qmtools
from qmtools import synthetic as syn
from oracle import basis as ob


def test_import_needs_no_gpu():
    import importlib
    m = importlib.reload(qmtools)
    assert hasattr(m, "QMTools")


def test_molecule_almos_and_units(basis, sample_molecule):
    mol = sample_molecule
    assert mol.natoms == 12 and mol.norbs == 162
    tabs = ob.reference_tables(qmtools.BASIS_CCPVDZ)
    assert np.array_equal(mol.ALMOs, ob.almo_table(mol.types, tabs))
    assert mol.qtot == 35 + 2 * 17 + 6 * 6 + 3
    assert mol.coords.dtype == np.float32


def test_unsupported_element_raises(basis):
    with pytest.raises((IndexError, KeyError)):
        qmtools.Molecule([[19, 0.0, 0.0, 0.0]], np.zeros((1, 1)), basis)
    with pytest.raises(IndexError):
        # Z=26 has an f shell: the reference's m table has no L=3 row
        qmtools.Molecule([[26, 0.0, 0.0, 0.0]], np.zeros((1, 1)), basis)


def test_grid_shape_rules():
    with pytest.raises(ValueError):
        qmtools.Grid((1, 10, 16, 16), 0.1)
    g = qmtools.Grid((16, 24, 32), 0.1)
    assert g.shape == (1, 16, 24, 32) and g.GPUblocks == (2, 3, 4)
    assert g.npts == 16 * 24 * 32
    assert abs(g.step - np.float32(0.1 * qmtools.ANG2BOR)) == 0
    assert g.origin["x"] == 0


def test_density_grid_geometry(sample_molecule):
    g = qmtools.Grid.DensityGrid(sample_molecule, 0.1, 2.0)
    c = sample_molecule.coords
    assert all(s % 8 == 0 for s in g.space_shape())
    assert np.isclose(g.origin["x"], c[:, 0].min() - 2.0 * qmtools.ANG2BOR)
    ext = (c.max(axis=0) - c.min(axis=0)) + 4.0 * qmtools.ANG2BOR
    assert np.all(np.array(g.space_shape()) * g.step >= ext - 1e-4)
    e = qmtools.Grid.emptyAs(g, nfields=2)
    assert e.shape == (2,) + g.space_shape() and e.step == g.step


def test_bin_roundtrip(tmp_path, sample_molecule):
    g = qmtools.Grid((1, 8, 16, 24), 0.2, [1.0, -2.0, 0.5])
    g.qube = np.random.default_rng(0).standard_normal(g.shape).astype(np.float32)
    f = tmp_path / "g.bin"
    g.SaveBIN(str(f), mol=sample_molecule)
    raw = f.read_bytes()
    (natm,) = struct.unpack_from("i", raw, 0)
    assert natm == 12
    assert struct.unpack_from("i", raw, 4)[0] == int(sample_molecule.types[0])
    h = qmtools.Grid.LoadBIN(str(f))
    assert h.shape == g.shape and h.step == g.step
    assert h.origin["y"] == np.float32(-2.0)
    assert np.array_equal(h.qube, g.qube)
    g.SaveBINmulti(str(tmp_path / "m"))
    assert (tmp_path / "m-0.bin").read_bytes()[4 + 28:] == raw[4 + 16 * 12 + 28:]


def test_pickle_save_load(tmp_path):
    g = qmtools.Grid((1, 8, 8, 8), 0.3, [0.1, 0.2, 0.3])
    g.qube[:] = 3.0
    g.Save(str(tmp_path / "g.pkl"))
    d = pickle.load(open(tmp_path / "g.pkl", "rb"))
    assert set(d) == {"shape", "origin", "step", "lattice", "qube"}
    h = qmtools.Grid.Load(None, str(tmp_path / "g.pkl"))
    assert np.array_equal(h.qube, g.qube) and h.origin["z"] == np.float32(0.3)


def test_synthetic_configs_are_seeded(basis):
    a = syn.config_molecule("c1")
    b = syn.config_molecule("c1")
    assert np.array_equal(a.coords_bohr, b.coords_bohr)
    assert sorted(a.types.tolist()) == sorted([6] * 10 + [1] * 14 + [7] * 3 + [8] * 3)
    d = np.sqrt(((a.coords_bohr[:, None] - a.coords_bohr[None]) ** 2).sum(-1))
    assert d[np.triu_indices(30, 1)].min() >= 1.8
    c0 = syn.config_molecule("c0")
    assert sorted(c0.types.tolist()) == [1] * 6 + [6] * 2
    m = c0.molecule(basis, qmtools.Molecule)
    assert m.norbs == 58
    S = syn.overlap(m.coords, m.ALMOs, basis.alphas, basis.coeffs)
    assert abs(np.sum(m.dm.astype(np.float64) * S) - 7) < 1e-5


def test_batch_and_stream_generators():
    mols = syn.batch_molecules(count=4)
    assert len(mols) == 4
    for m in mols:
        assert 5 <= len(m.types) <= 60 and all(s % 8 == 0 for s in m.grid_shape)
    st = syn.serving_stream(200.0, 5)
    t = [x for x, _ in st]
    assert all(t[i] < t[i + 1] for i in range(4))


def test_fft_candidates_are_nice_and_long_enough():
    from qmtools.autotune import fft_candidates
    for n in (24, 40, 64, 68, 136, 160):
        c = fft_candidates(n)
        assert c and all(m >= 2 * n for m in c)
        for m in c:
            k = m
            for r in (2, 3, 5, 7):
                while k % r == 0:
                    k //= r
            assert k == 1


def test_tuner_without_measuring_uses_defaults(tmp_path):
    """With measuring off the tuner returns the defaults without touching the GPU or the cache."""
    import types
    from qmtools.autotune import PATH_FUSED, PATH_STAGED, Tuner
    t = Tuner(path=tmp_path / "none.json", measure=False)
    t._device_key = lambda: "cpu-test"
    small = types.SimpleNamespace(norbs=100)
    big = types.SimpleNamespace(norbs=400)
    assert t.density_path(small, 4096, "fp16x3") == PATH_FUSED
    assert t.density_path(big, 4096, "fp16x3") == PATH_STAGED
    assert t.density_path(small, 4096, "tf32x3") == PATH_STAGED
    assert t.fft_length(40, small) == 80
    assert not (tmp_path / "none.json").exists()
