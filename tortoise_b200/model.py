"""Host-side model objects shaped like the reference's public API.

Region, Mesh, Band, ScatteringChannel, Material, MaterialStatus and
MaterialTimeStatus keep the reference's names and argument meaning
(include/Geometry/Structured/DirectSpace/Region.hpp, Mesh.hpp,
include/Physics/Material/Band.hpp, Material.hpp,
include/Physics/Scattering/ScatteringChannel.hpp,
include/Physics/Status/MaterialStatus.hpp, MaterialTimeStatus.hpp).  They
hold geometry and parameters only; every propagation goes through the CUDA
library bound in ``tortoise_b200.engine``.
"""
import hashlib
import os
import struct

import numpy as np

from .abi import BOSON, FERMION, IN, OUT, PackedProblem

__all__ = ["Region", "Mesh", "Band", "ScatteringChannel", "Material", "MaterialStatus",
           "MaterialTimeStatus", "IN", "OUT", "FERMION", "BOSON", "match_string",
           "random_points_reference"]

# Section-relative vertices of the two elements of a section
# (src/Geometry/Structured/DirectSpace/Mesh.cpp:48-84).
_VERT = np.array([[[0, 0], [1, 0], [1, 1]], [[0, 0], [0, 1], [1, 1]]], dtype=np.float64)


def match_string(pattern, candidate):
    """'*' / '?' wildcard match of src/Generics/Utilities/StringUtilities.cpp:44-61."""
    def rec(p, c):
        if p == len(pattern):
            return c == len(candidate)
        if pattern[p] == "*":
            for cc in range(c, len(candidate) + 1):
                if rec(p + 1, cc):
                    return True
            return False
        if c == len(candidate) or (pattern[p] != "?" and pattern[p] != candidate[c]):
            return False
        return rec(p + 1, c + 1)
    return rec(0, 0)


def random_points_reference(rng, ndim, n):
    """Uniform points in the reference simplex by the cut-and-fold of
    include/Geometry/GeometryCore/Point.hpp:44-68, drawn from a seeded numpy
    generator instead of the reference's unseeded Eigen::Random."""
    pts = rng.random((n, ndim))
    if ndim == 2:
        fold = pts[:, 0] + pts[:, 1] > 1.0
        pts[fold] = 1.0 - pts[fold]
    return pts


class Region:
    """Region<2>: origin plus two side vectors (the columns of gvec)."""

    def __init__(self, origin, sides):
        self.origin = np.asarray(origin, dtype=np.float64).reshape(2)
        s = np.asarray(sides, dtype=np.float64).reshape(2, 2)
        self.gvec = s.T.copy()  # columns are the sides


class Mesh:
    """Mesh<2>(region, relativeOrigin, relativeSize, nSecSplits)
    (src/Geometry/Structured/DirectSpace/Mesh.cpp:319-347)."""

    def __init__(self, region, rel_origin, rel_size, nsplit):
        self.region = region
        self.rel_origin = np.asarray(rel_origin, dtype=np.float64).reshape(2)
        self.rel_size = np.asarray(rel_size, dtype=np.float64).reshape(2)
        self.nsplit = (int(nsplit[0]), int(nsplit[1]))
        G = region.gvec
        self.origin = region.origin + (G[:, 0] * self.rel_origin[0] + G[:, 1] * self.rel_origin[1])
        gv = G * self.rel_size[None, :]
        self.dG = gv * (1.0 / np.array(self.nsplit, dtype=np.float64))[None, :]
        self.numberElements = 2 * self.nsplit[0] * self.nsplit[1]
        self.elemVolume = abs((self.dG[0, 0] * self.dG[1, 1] - self.dG[0, 1] * self.dG[1, 0]) / 2.0)

    @property
    def ne(self):
        return self.numberElements

    def vertices(self):
        """(Ne, 3, 2) absolute vertex coordinates (Mesh.cpp:488-494)."""
        e = np.arange(self.ne)
        s, par = e // 2, e % 2
        sx = (s % self.nsplit[0]).astype(np.float64)
        sy = (s // self.nsplit[0]).astype(np.float64)
        px = sx[:, None] + _VERT[par][:, :, 0]
        py = sy[:, None] + _VERT[par][:, :, 1]
        x = self.origin[0] + (self.dG[0, 0] * px + self.dG[0, 1] * py)
        y = self.origin[1] + (self.dG[1, 0] * px + self.dG[1, 1] * py)
        return np.stack([x, y], axis=-1)

    def function(self, fn):
        """Function<2>(mesh, lambda): nodal samples -> linear-form coefficients
        (src/Geometry/Structured/FunctionSpace/Function.cpp:60-68).
        ``fn(kx, ky)`` is evaluated on arrays; scalars give constant functions."""
        v = self.vertices()
        if callable(fn):
            nodal = np.asarray(fn(v[..., 0], v[..., 1]), dtype=np.float64)
            nodal = np.broadcast_to(nodal, (self.ne, 3)).copy()
        else:
            nodal = np.full((self.ne, 3), float(fn))
        return nodal_to_linform(nodal)


def read_scatt_indices(path, nlegs, nsplit=None):
    """A "<scatteringName>.scattIndices" file (ScatteringChannel.cpp:421-458):
    int32 mesh splits of every leg, uint64 count, then per tuple nlegs int32
    element ids and an int32 umklapp column.  Returns (ids[n, nlegs],
    umklapp[n]) or (None, None) when the splits differ from nsplit."""
    raw = open(path, "rb").read()
    head = np.frombuffer(raw, dtype="<i4", count=2 * nlegs)
    if nsplit is not None and list(head) != [int(x) for x in nsplit]:
        return None, None
    (n,) = struct.unpack_from("<Q", raw, 8 * nlegs)
    rec = np.frombuffer(raw, dtype="<i4", count=n * (nlegs + 1), offset=8 * nlegs + 8).reshape(n, nlegs + 1)
    return np.ascontiguousarray(rec[:, :nlegs]), np.ascontiguousarray(rec[:, nlegs])


def nodal_to_linform(nodal):
    nodal = np.asarray(nodal, dtype=np.float64).reshape(-1, 3)
    out = nodal.copy()
    out[:, 1] = nodal[:, 1] - nodal[:, 0]
    out[:, 2] = nodal[:, 2] - nodal[:, 0]
    return out.reshape(-1)


def linform_to_nodal(lin):
    lin = np.asarray(lin, dtype=np.float64).reshape(-1, 3)
    out = lin.copy()
    out[:, 1] = lin[:, 1] + lin[:, 0]
    out[:, 2] = lin[:, 2] + lin[:, 0]
    return out


class Band:
    """Band<2> (include/Physics/Material/Band.hpp:49-113)."""

    def __init__(self, name, charge, statistics, mesh, dispersion):
        self.name = name
        self.charge = float(charge)
        self.statistics = float(statistics)
        self.mesh = mesh
        self.dispersion_coeffs = mesh.function(dispersion)
        self.absoluteErrorTolerance = 1.0e-3
        self.relativeErrorTolerance = 1.0e-3
        self.penalisationUnphysicalPopulation = 0.0
        self.constrained = False
        self.constrainedPopulation = None
        self.drift_velocity = (0.0, 0.0)

    def constrain(self, population):
        """Band::constrained with its constrainedPopulation (Band.hpp:70-74):
        an array of Ne*3 linear-form coefficients (time-independent, e.g. a
        reservoir) or a callable t -> coefficients (e.g. a laser pulse); a
        callable is evaluated by the integrator at every enforce time and drives
        the time-step veto, as the reference's std::function does."""
        self.constrained = True
        if callable(population):
            self.constrainedPopulation = population
        else:
            self.constrainedPopulation = np.ascontiguousarray(population, dtype=np.float64)

    def population_at(self, t):
        """constrainedPopulation(t) (the array itself when time-independent)."""
        p = self.constrainedPopulation
        return np.ascontiguousarray(p(t) if callable(p) else p, dtype=np.float64)


class ScatteringChannel:
    """ScatteringChannel<2,L> parameters (ScatteringChannel.hpp:54-102).  The
    Monte-Carlo table is an explicit seeded input (the reference redraws it
    from std::rand at every propagation, MaterialTimeStatus.cpp:104)."""

    def __init__(self, material, band_numbers, directions, mc_seed):
        self.material = material
        self.nlegs = len(band_numbers)
        self.legBandNumber = [int(b) for b in band_numbers]
        self.legDirection = [int(d) for d in directions]
        self.amplitude = 1.0
        # ScatteringChannel::functAmplitude (ScatteringChannel.hpp:74): None
        # is the reference's default 1; else a vectorised callable
        # barycentres[n, nlegs, 2] -> factors[n] (one per tuple, at its
        # elements' barycentres)
        self.functAmplitude = None
        self.numMCPoints = material.defaultNMCPointsScatterings
        self.minimumDeterminant = material.defaultMinimumDeterminantScatterings
        self.scattElemeThreshold = material.defaultScattElemeThresholdScatterings
        self.umklappUnitVectors = np.zeros((1, 2))
        self.mc_seed = int(mc_seed)
        self.tuples = None
        self.tuple_umklapp = None
        self.constructMCPoints()

    def scatteringName(self):
        m = self.material
        ins = "".join("(" + m.band_names[b] + ")" for b, d in zip(self.legBandNumber, self.legDirection) if d > 0)
        outs = "".join("(" + m.band_names[b] + ")" for b, d in zip(self.legBandNumber, self.legDirection) if d < 0)
        return "[" + ins + "]-[" + outs + "]"

    def content_hash(self):
        """SHA-256 of every input the tuple list depends on: region, the legs'
        meshes, dispersions and directions, the umklapp table, the survival
        points, minimum determinant, threshold and amplitude.  The
        reference's cache only checks the mesh splits; this digest, kept in
        a side file, also catches a changed dispersion, table or threshold."""
        m = self.material
        h = hashlib.sha256()
        h.update(np.asarray(m.region.origin, dtype=np.float64).tobytes())
        h.update(np.asarray(m.region.gvec, dtype=np.float64).tobytes())
        for b, d in zip(self.legBandNumber, self.legDirection):
            band = m.bands[b]
            mesh = band.mesh
            h.update(struct.pack("<ii", int(mesh.nsplit[0]), int(mesh.nsplit[1])))
            h.update(np.asarray(mesh.rel_origin, dtype=np.float64).tobytes())
            h.update(np.asarray(mesh.rel_size, dtype=np.float64).tobytes())
            h.update(np.ascontiguousarray(band.dispersion_coeffs, dtype=np.float64).tobytes())
            h.update(struct.pack("<id", int(d), float(band.statistics)))
        h.update(np.ascontiguousarray(self.umklappUnitVectors, dtype=np.float64).tobytes())
        h.update(np.ascontiguousarray(self.mc_points_precalc, dtype=np.float64).tobytes())
        h.update(struct.pack("<ddd", float(self.minimumDeterminant), float(self.scattElemeThreshold),
                             float(self.amplitude)))
        return h.hexdigest()

    def findUmklappVectors(self, n):
        """All (2n+1)^2 test vectors are kept (ScatteringChannel.cpp:194-215)."""
        r = range(-n, n + 1)
        self.umklappUnitVectors = np.array([[i, j] for i in r for j in r], dtype=np.float64)
        return len(self.umklappUnitVectors) != 0

    def constructMCPoints(self, seed=None):
        """Rows: (L-2) reference-triangle points then one [0,1] coordinate
        (ScatteringChannel.cpp:677-688); a second independent table stands in
        for the per-tuple draws of the survival test (IntegratorCore.hpp:382-388)."""
        if seed is not None:
            self.mc_seed = int(seed)
        L, n = self.nlegs, self.numMCPoints
        for which, off in (("mc_points", 0), ("mc_points_precalc", 1)):
            rng = np.random.default_rng([self.mc_seed, off])
            cols = [random_points_reference(rng, 2, n) for _ in range(L - 2)]
            cols.append(random_points_reference(rng, 1, n))
            setattr(self, which, np.ascontiguousarray(np.concatenate(cols, axis=1)))


class Material:
    """Material<2> (include/Physics/Material/Material.hpp:58-188)."""

    def __init__(self, matID, region):
        self.matID = matID
        self.region = region
        self.bands = []
        self.band_names = []
        self.channels = []
        self.defaultNMCPointsScatterings = 50
        self.defaultMinimumDeterminantScatterings = 1.0e-9
        self.defaultScattElemeThresholdScatterings = 1.0e-9
        self._mc_seed_base = 0x5EED
        self._engine = None

    # -- bands -----------------------------------------------------------
    def addBand(self, t_id, t_charge, t_statistics, t_mesh, t_dispersion):
        assert t_mesh.region is self.region
        b = Band(t_id, t_charge, t_statistics, t_mesh, t_dispersion)
        self.bands.append(b)
        self.band_names.append(t_id)
        self._engine = None
        return b

    def __getitem__(self, name):
        return self.bands[self.id(name)]

    def id(self, name):
        return self.band_names.index(name)

    def matchListId(self, wildcard):
        return [n for n in self.band_names if match_string(wildcard, n)]

    @property
    def meshes(self):
        out = []
        for b in self.bands:
            if all(m is not b.mesh for m in out):
                out.append(b.mesh)
        return out

    # -- channels --------------------------------------------------------
    def addScatteringChannel(self, band_names, directions):
        c = ScatteringChannel(self, [self.id(n) for n in band_names], directions,
                              self._mc_seed_base + len(self.channels))
        self.channels.append(c)
        self._engine = None
        return c

    def addScatteringChannelsWildcards(self, band_names, directions, numUmklappSteps):
        """Band combinations with exchange / time-reversal deduplication
        (src/Physics/Material/Material.cpp:209-364).  Channels whose tuple list
        turns out empty contribute nothing (the reference pops them)."""
        L = len(band_names)
        lists = [self.matchListId(w) for w in band_names]
        added = []

        def groups(names, dirs):
            gi = sorted(n for n, d in zip(names, dirs) if d == IN)
            go = sorted(n for n, d in zip(names, dirs) if d != IN)
            return gi, go

        import itertools
        for combo in itertools.product(*lists):
            if L == 2:
                found = False
                for c in self.channels:
                    if c.nlegs != 2:
                        continue
                    have = sorted(self.band_names[b] for b in c.legBandNumber)
                    if have == sorted(combo) and directions[0] * directions[1] == c.legDirection[0] * c.legDirection[1]:
                        found = True
                        break
            else:
                gi, go = groups(combo, directions)
                found = False
                for c in self.channels:
                    if c.nlegs != L:
                        continue
                    ci, co = groups([self.band_names[b] for b in c.legBandNumber], c.legDirection)
                    if (len(gi) == len(ci) and gi == ci and go == co) or (len(gi) == len(co) and gi == co and go == ci):
                        found = True
                        break
            if found:
                continue
            c = self.addScatteringChannel(list(combo), directions)
            c.findUmklappVectors(numUmklappSteps)
            added.append(c)
        return added

    # -- analysis (Material.cpp:396-410) -----------------------------------
    def scatteringChannelMatchList(self, band_names_wildcards, directions):
        """Channels whose ordered legs match the wildcards and directions
        exactly (Material.cpp:124-162)."""
        L = len(band_names_wildcards)
        out = []
        for i, c in enumerate(self.channels):
            if c.nlegs != L or list(c.legDirection) != list(directions):
                continue
            if all(match_string(w, self.band_names[b]) for w, b in zip(band_names_wildcards, c.legBandNumber)):
                out.append(i)
        return out

    def scatteringRates(self, band_names_wildcards, directions, status, bandName):
        """Material::scatteringRates<L> (Material.cpp:396-402): out-scattering
        rates of band bandName from the matching channels, on the GPU."""
        eng = self.engine()
        b = self.id(bandName)
        offs, _ = self.band_offsets()
        out = np.zeros(self.bands[b].mesh.ne * 3)
        for ch in self.scatteringChannelMatchList(band_names_wildcards, directions):
            for leg, lb in enumerate(self.channels[ch].legBandNumber):
                if lb == b:
                    out += eng.scattering_rates(status.vec, ch, leg)[offs[b]:offs[b] + out.size]
        return out

    def selectivePropagation(self, band_names_wildcards, directions, status, bandName):
        """Material::selectivePropagation<L> (Material.cpp:404-410)."""
        eng = self.engine()
        tot = np.zeros(status.vec.size)
        for ch in self.scatteringChannelMatchList(band_names_wildcards, directions):
            tot += eng.channel_propagate(ch, status.vec)
        b = self.id(bandName)
        offs, _ = self.band_offsets()
        return tot[offs[b]:offs[b] + self.bands[b].mesh.ne * 3]

    # -- packing ---------------------------------------------------------
    def pack(self):
        return PackedProblem(self.region, self.meshes, self.bands, self.channels)

    def band_offsets(self):
        off, out = 0, []
        for b in self.bands:
            out.append(off)
            off += b.mesh.ne * 3
        return out, off

    # -- tuple cache (ScatteringChannel.cpp:421-458, 516-534) ----------------
    def cache_path(self, directory, ch):
        return os.path.join(directory, self.channels[ch].scatteringName() + ".scattIndices")

    def load_tuple_cache(self, directory):
        """Reads "<scatteringName>.scattIndices" of every channel whose file
        exists, whose header matches its legs' mesh splits (the reference's
        test) and whose side file "<...>.sha256" matches content_hash() (a
        file without a side file, e.g. one the reference wrote, is trusted as
        the reference trusts it).  Returns the channels loaded."""
        loaded = []
        for ch, c in enumerate(self.channels):
            path = self.cache_path(directory, ch)
            if not os.path.exists(path):
                continue
            side = path + ".sha256"
            if os.path.exists(side) and open(side).read().strip() != c.content_hash():
                continue
            ns = [self.bands[b].mesh.nsplit[k] for b in c.legBandNumber for k in (0, 1)]
            ids, umk = read_scatt_indices(path, c.nlegs, ns)
            if ids is None:
                continue
            c.tuples, c.tuple_umklapp = ids, umk
            loaded.append(ch)
        self._engine = None
        return loaded

    def save_tuple_cache(self, directory, engine=None):
        """Writes every channel's tuple list in the reference's format (with
        the content digest in a side file)."""
        eng = engine or self.engine()
        os.makedirs(directory, exist_ok=True)
        for ch, c in enumerate(self.channels):
            path = self.cache_path(directory, ch)
            eng.write_scatt_indices(ch, path)
            with open(path + ".sha256", "w") as fh:
                fh.write(c.content_hash() + "\n")

    def engine(self, **opts):
        """The CUDA handle for this material (built on first use)."""
        from .engine import Engine
        if self._engine is None or opts:
            self._engine = Engine(self, **opts)
        return self._engine


class MaterialStatus:
    """MaterialStatus<2>: the concatenated band populations
    (include/Physics/Status/MaterialStatus.hpp:46-140)."""

    def __init__(self, material, vec=None):
        self.material = material
        self.offsets, self.ndofs = material.band_offsets()
        self.vec = np.zeros(self.ndofs) if vec is None else np.ascontiguousarray(vec, dtype=np.float64).copy()

    def __getitem__(self, name):
        b = self.material.id(name)
        o = self.offsets[b]
        return self.vec[o:o + self.material.bands[b].mesh.ne * 3]

    def __setitem__(self, name, coeffs):
        self[name][:] = coeffs

    def copy(self):
        return MaterialStatus(self.material, self.vec)

    def setToEquilibrium(self, temperature, chemicalPotentialFermions, chemicalPotentialBosons):
        """MaterialStatus.cpp:212-220: Fermi-Dirac / Bose-Einstein of the
        dispersion, evaluated nodally (Function.cpp:75-89)."""
        for b in self.material.bands:
            e = linform_to_nodal(b.dispersion_coeffs)
            if b.statistics == FERMION:
                nod = 1.0 / (np.exp((e - chemicalPotentialFermions) / temperature) + 1.0)
            else:
                nod = 1.0 / (np.exp((e - chemicalPotentialBosons) / temperature) - 1.0)
            self[b.name] = nodal_to_linform(nod)

    def propagate(self):
        """MaterialStatus::propagate (MaterialStatus.cpp:146-161) on the GPU,
        plus the drift term of bands with a nonzero drift velocity."""
        return MaterialStatus(self.material, self.material.engine().rhs(self.vec))

    def relativeError(self, population):
        return self.material.engine().relative_error(self.vec, population.vec)

    # -- I/O: MaterialStatus::save / load, declared in the reference
    # (MaterialStatus.hpp:131-132) but never defined there.  File: magic
    # "TBMS1", band count, then per band its name, element count and the
    # 3 x elements linear-form coefficients (little-endian FP64).
    def save(self, fileName):
        with open(fileName, "wb") as fh:
            fh.write(b"TBMS1")
            fh.write(struct.pack("<i", len(self.material.bands)))
            for b, band in enumerate(self.material.bands):
                name = band.name.encode()
                fh.write(struct.pack("<i", len(name)) + name)
                fh.write(struct.pack("<q", band.mesh.ne))
                fh.write(np.ascontiguousarray(self[band.name], dtype="<f8").tobytes())

    def load(self, fileName):
        with open(fileName, "rb") as fh:
            if fh.read(5) != b"TBMS1":
                raise ValueError("%s is not a saved MaterialStatus" % fileName)
            (nb,) = struct.unpack("<i", fh.read(4))
            if nb != len(self.material.bands):
                raise ValueError("saved status has %d bands, the material %d" % (nb, len(self.material.bands)))
            for band in self.material.bands:
                (ln,) = struct.unpack("<i", fh.read(4))
                name = fh.read(ln).decode()
                (ne,) = struct.unpack("<q", fh.read(8))
                if name != band.name or ne != band.mesh.ne:
                    raise ValueError("saved band %s (%d elements) does not match %s (%d)"
                                     % (name, ne, band.name, band.mesh.ne))
                self[band.name] = np.frombuffer(fh.read(24 * ne), dtype="<f8")
        return self

    def scatteringRates(self):
        """MaterialStatus::scatteringRates (MaterialStatus.cpp:170-187): the
        out-scattering rate of every band from every channel, on the GPU."""
        return MaterialStatus(self.material, self.material.engine().scattering_rates(self.vec))


class MaterialTimeStatus:
    """MaterialTimeStatus<2>: dense-output trajectory
    (include/Physics/Status/MaterialTimeStatus.hpp)."""

    def __init__(self, status, time0=0.0):
        self.material = status.material
        self.times = [float(time0)]
        self.statuses = [status.copy()]
        self.stats = None

    def __len__(self):
        return len(self.times)

    def __getitem__(self, i):
        return self.statuses[i]

    def back(self):
        return self.statuses[-1]

    def propagate(self, finalTime, denseStep, max_dense=None):
        """DP5(4) from the last stored time to finalTime
        (MaterialTimeStatus.cpp:102-137), integrated entirely on the GPU."""
        eng = self.material.engine()
        res = eng.dp45(self.statuses[-1].vec, self.times[-1], finalTime, denseStep, max_dense=max_dense)
        for t, v in zip(res["dense_t"], res["dense"]):
            self.times.append(float(t))
            self.statuses.append(MaterialStatus(self.material, v))
        self.stats = res
        return res
