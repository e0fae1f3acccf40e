"""Golden traces of the reference's GA engine (qmtools/GAEngine.py), for tests/test_ga_engine.py.

The reference engine is plain Python + NumPy, so this script imports it straight from the
reference sources (only where they are present) and records, from fixed NumPy seeds: random
elements, crossover, mutation (amounts 0.5 and 1.0), serialisation bytes, option parsing and a
three-generation run on the engine's toy sine-series problem (fitnesses per generation, the
restart file and the next population).  The committed tests/golden/ga_engine.npz was produced by

    python tests/golden/make_ga_golden.py [path/to/reference/qmtools/GAEngine.py]
"""
import importlib.util
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

DEFAULT_SRC = "/root/reference/qmtools/GAEngine.py"
OUT = Path(__file__).resolve().parent / "ga_engine.npz"


def load(src):
    spec = importlib.util.spec_from_file_location("ref_gaengine", src)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def refdata():
    xs = np.linspace(0.0, 3.0, 41)
    return np.stack([xs, 0.7 * np.sin(xs) - 0.3 * np.sin(3 * xs)], axis=1)


def traces(mod, workdir):
    out = {}
    E, GA = mod.GAElement, mod.GA
    np.random.seed(11)
    a = E.Random(pscale=2.0)
    b = E.Random(pscale=2.0)
    out["rand_a"], out["rand_b"] = a.params.copy(), b.params.copy()
    r = E.Mix(a, b)
    out["mix"] = r.params.copy()
    r.Mutate(0.5, 0.1)
    out["mutate_05"] = r.params.copy()
    r.Mutate(1.0, 0.1)
    out["mutate_10"] = r.params.copy()
    a.fitness = -1.25
    out["serialized"] = np.frombuffer(a.Serialize(), dtype=np.uint8).copy()
    argv = ["train.py", "--populationSize", "8", "--mutationRate", "0.5", "--keepbest", "1", "--logfile", "x.log"]
    opts = GA.ReadParameters(argv)
    out["opts"] = np.array([repr(sorted(opts.items()))])
    # a short run
    np.random.seed(12)
    ga = GA(populationSize=8, mutationRate=0.5, mutationSize=0.2, rerands=1, keepbest=True,
            logfile=os.path.join(workdir, "ga.log"), rstfile=os.path.join(workdir, "ga.restart.bin"))
    ga.elementTemplate = E
    ga.Initialize()
    fits = []
    for _ in range(3):
        ga.Evolve(refdata=refdata())
        fits.append(ga.fits.copy())
    out["run_fits"] = np.array(fits)
    out["run_offspring"] = np.array([e.params for e in ga.offspring])
    out["run_restart"] = np.frombuffer(Path(ga.rstfile).read_bytes(), dtype=np.uint8).copy()
    ga.flog.close()
    # restart: a new engine seeded alike, loading the file
    np.random.seed(13)
    ga2 = GA(populationSize=8, logfile=os.path.join(workdir, "ga2.log"), restart=ga.rstfile)
    ga2.elementTemplate = E
    ga2.Initialize()
    out["restart_offspring"] = np.array([e.params for e in ga2.offspring])
    ga2.flog.close()
    return out


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SRC
    mod = load(src)
    with tempfile.TemporaryDirectory() as td:
        out = traces(mod, td)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
