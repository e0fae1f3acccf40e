"""Genetic-algorithm engine of the QMTools training scripts (drop-in for qmtools.GAEngine).

Same classes, methods, keyword options, log/restart files and random-number use as the
reference engine (qmtools/GAEngine.py), so that `scripts/train-singleshot.py` runs unchanged
and a seeded run draws the same numbers in the same order:

* GAElement (qmtools/GAEngine.py:8-134): parameters + fitness, `struct` serialisation with the
  element's format ('d' here, 'f' for the float32 automaton), uniform-mask crossover, masked
  mutation, and a toy sine-series Evaluate.
* GA (qmtools/GAEngine.py:139-365): population, soft rank selection
  p_i ~ exp(-ln(10) i / n) over the sorted population, crossover, mutation, optional elitism,
  random immigrants, a restart file written every generation and a log of best/worst/mean.

Two behaviours of the reference are kept as they are, because seeded runs must match:
GAElement.Mutate zeroes its mask again right after setting it (for amount < 1 no parameter
changes), and the second parent of a pair is drawn from the index list with the first parent's
index replaced by 0 (so index 0 may be drawn twice as often, and may equal the first parent).
"""
import builtins
import struct

import numpy


class GAElement:
    """Base element: override Random, Serialize/Deserialize, Mix, Mutate and Evaluate."""

    def __init__(self):
        self.fitness = -9999
        self.params = []
        self._dnasize = 0
        self._precision = 8
        self._format = 'd'

    def Random(**kwargs):
        pscale = kwargs.get('pscale', 1.0)
        e = GAElement()
        e._dnasize = 5
        e.params = pscale * (2 * numpy.random.random(e._dnasize) - 1)
        return e

    def Serialize(self):
        """Bytes of every parameter, then the fitness, each packed with the element's format."""
        packed = [struct.pack(self._format, v) for v in self.params]
        packed.append(struct.pack(self._format, self.fitness))
        return b''.join(packed)

    def Deserialize(self, barray):
        """Reads len(params) values and the fitness from `barray`; returns the bytes used."""
        w = self._precision
        n = self.params.shape[0]
        for i in range(n):
            self.params[i] = struct.unpack(self._format, barray[i * w:(i + 1) * w])[0]
        self.fitness = struct.unpack(self._format, barray[n * w:(n + 1) * w])[0]
        print('GAElement loaded [fitness={}]'.format(self.fitness))
        return (n + 1) * w

    def Mix(a, b):
        """Uniform crossover: each parameter from `a` where a uniform draw is < 0.5, else `b`."""
        r = a.__class__()
        r.params = numpy.copy(a.params)
        r._dnasize = a._dnasize
        draw = numpy.random.random(a.params.shape[0])
        from_a = numpy.where(draw < 0.5, 1, 0).astype(r.params.dtype)
        from_b = (1 - from_a).astype(r.params.dtype)
        r.params = from_a * a.params + from_b * b.params
        return r

    def Mutate(self, amount, mscale, **kwargs):
        dt = self.params.dtype
        mutagen = ((2 * numpy.random.random(self._dnasize) - 1) * mscale).astype(dt)
        mask = numpy.random.random(self._dnasize).astype(dt)
        # as the reference: the mask is set to 1 where <= amount, then everything > amount
        # (those ones included when amount < 1) is set to 0
        mask[mask <= amount] = 1
        mask[mask > amount] = 0
        self.params += mutagen * mask

    def Evaluate(self, **kwargs):
        refdata = kwargs.get('refdata', None)
        if refdata is None:
            print('invalid refdata!')
            return 0
        xs, ys = refdata[:, 0], refdata[:, 1]
        yp = ys * 0
        for i in range(self.params.shape[0]):
            yp += self.params[i] * numpy.sin(xs * (i + 1))
        self.fitness = -numpy.mean(numpy.abs(yp - ys))
        return self.fitness


class GA:

    PARAMS = {
        'float': ['mutationRate', 'mutationSize', 'pscale'],
        'int': ['populationSize', 'rerands', 'rstfreq'],
        'bool': ['keepbest'],
    }

    def ProcessParameter(name, value):
        """Converts a command-line value to the type its option has (strings otherwise)."""
        for typename, names in GA.PARAMS.items():
            if name in names:
                return vars(builtins)[typename](value)
        return value

    def ReadParameters(plist):
        """`--name value` pairs of an argument list -> keyword options."""
        opts = {}
        for i, item in enumerate(plist):
            if item.startswith('--'):
                opts[item[2:]] = GA.ProcessParameter(item[2:], plist[i + 1])
        return opts

    def __init__(self, **kwargs):
        self.populationSize = kwargs.get('populationSize', 128)
        self.keepbest = kwargs.get('keepbest', False)
        self.rerands = kwargs.get('rerands', 1)
        self.mutationRate = kwargs.get('mutationRate', 0.02)
        self.mutationSize = kwargs.get('mutationSize', 0.10)
        self.pscale = kwargs.get('pscale', 1.0)
        self.logfile = kwargs.get('logfile', "ga.log")
        self.outfile = kwargs.get('outfile', "ga.out.bin")
        self.rstfile = kwargs.get('rstfile', "ga.restart.bin")
        self.rstfreq = kwargs.get('rstfreq', 1)
        self.restart = kwargs.get('restart', None)
        self.indexes = numpy.arange(self.populationSize)
        self.elementTemplate = None
        self.elementInitDict = {}
        self.population = None
        self.offspring = None
        self.fits = []
        self.generation = 0

    def _initer(self):
        d = dict(self.elementInitDict)
        d['pscale'] = self.pscale
        return d

    def Initialize(self, noLog=False):
        self.offspring = [self.elementTemplate.Random(**self._initer()) for _ in range(self.populationSize)]
        if not noLog:
            self.flog = open(self.logfile, "w")
        if self.restart is not None:
            with open(self.restart, "rb") as f:
                barray = f.read()
            for e in self.offspring:
                barray = barray[e.Deserialize(barray):]
            # the restart holds an evaluated population: breed the next one from it
            self.population = self.offspring
            self.fits = numpy.asarray([e.fitness for e in self.population])
            self.Reproduce()

    def Evolve(self, **kwargs):
        """One generation: evaluate, report, write the restart file, reproduce."""
        debug = kwargs.get('debug', False)
        self.population = list(self.offspring[:self.populationSize])
        self.fits = numpy.zeros(self.populationSize)
        for i, atm in enumerate(self.population):
            self.fits[i] = atm.Evaluate(**kwargs)
            if debug:
                print("generation[{}] element[{}] fitness {}".format(self.generation, i, self.fits[i]))
        fitmax, fitmin, fitmean = numpy.max(self.fits), numpy.min(self.fits), numpy.mean(self.fits)
        print("generation {0}: best {1:8.5f} -- worst {2:8.5f} -- mean {3:8.5f}".format(
            self.generation, fitmax, fitmin, fitmean))
        with open(self.rstfile, "wb") as f:
            for e in self.population:
                f.write(e.Serialize())
        self.generation += 1
        self.flog.write("{} {} {}\n".format(fitmax, fitmin, fitmean))
        self.flog.flush()
        self.Reproduce()

    def Reproduce(self):
        """Next population from the evaluated one (best first after sorting by fitness)."""
        order = numpy.argsort(-self.fits)
        self.fits = self.fits[order]
        pop = [self.population[i] for i in order]
        best = numpy.argmax(self.fits)
        n = self.populationSize
        idx = numpy.arange(n)
        k = numpy.log(10.0) / len(pop)
        prob = numpy.exp(-k * numpy.arange(len(pop)))
        prob /= numpy.sum(prob)
        first = numpy.random.choice(idx, replace=True, size=n, p=prob)
        second = first * 0
        for i in range(n):
            # the first parent's slot holds 0 instead of its index (reference behaviour)
            candidates = numpy.where(idx != first[i], idx, 0)
            second[i] = numpy.random.choice(candidates, p=prob)
        self.offspring = [self.elementTemplate.Mix(pop[a], pop[b]) for a, b in zip(first, second)]
        for atm in self.offspring:
            if numpy.random.random() < self.mutationRate:
                atm.Mutate(self.mutationSize, self.pscale)
        if self.keepbest:
            self.offspring[0] = pop[best]
        for i in range(self.rerands):
            self.offspring[n - 1 - i] = self.elementTemplate.Random(**self._initer())
