"""Synthetic materials with the shapes of the benchmark configurations.

k-space square [-1,1]^2 split into N x N sections (2 N^2 triangles); bands are
sampled at the P1 vertices like Function<2>(mesh, lambda) does.  Electron bands:
parabola E=|k|^2/2, Dirac cone E=|k|+0.5, heavy hole E=-|k|^2/6-0.3.  Optical
phonon branches are dispersionless boson bands on the same mesh.  Channels are
created with Material::addScatteringChannelsWildcards exactly as the reference
tutorials do: e-e {el:*,el:*,el:*,el:*} {in,in,out,out} and e-ph
{el:*,pn:*,el:*} {in,in,out}.

Initial state: Fermi-Dirac(kT, mu=0.3) plus a seeded Gaussian hot-carrier bump
(sigma 0.15, amplitude 0.3) multiplied by (1-f_FD) so that 0 <= f <= 1 holds
(a bare 0.3 bump on f_FD ~ 0.95 would give f > 1); phonons start at
Bose-Einstein(kT_ph).  All draws come from numpy PCG64 with an explicit seed.
"""
import numpy as np

from .model import BOSON, FERMION, IN, OUT, Material, MaterialStatus, Mesh, Region, linform_to_nodal, nodal_to_linform

DISPERSIONS = {
    "P": lambda kx, ky: 0.5 * (kx * kx + ky * ky),
    "D": lambda kx, ky: np.sqrt(kx * kx + ky * ky) + 0.5,
    "H": lambda kx, ky: -(kx * kx + ky * ky) / (2.0 * 3.0) - 0.3,
}


def build_material(N, electron_bands=("P",), phonon_energies=(), ee=True, eph=True,
                   field=(0.0, 0.0), ee_amplitude=1.0, eph_amplitude=1.0, n_mc=50,
                   rtol=1e-6, atol=1e-9, phonon_bath=False, kT_phonon=0.05, mc_seed=0x5EED,
                   mesh_nsplit=None):
    region = Region((-1.0, -1.0), ((2.0, 0.0), (0.0, 2.0)))
    ns = mesh_nsplit or (N, N)
    mesh = Mesh(region, (0.0, 0.0), (1.0, 1.0), ns)
    mat = Material("synthetic", region)
    mat.defaultNMCPointsScatterings = n_mc
    mat._mc_seed_base = mc_seed
    mat._mesh_keep = mesh
    for name in electron_bands:
        b = mat.addBand("el:" + name, -1.0, FERMION, mesh, DISPERSIONS[name])
        b.relativeErrorTolerance = rtol
        b.absoluteErrorTolerance = atol
        b.drift_velocity = (b.charge * field[0], b.charge * field[1])
    for i, w in enumerate(phonon_energies):
        b = mat.addBand("pn:%d" % i, 0.0, BOSON, mesh, float(w))
        b.relativeErrorTolerance = rtol
        b.absoluteErrorTolerance = atol
        if phonon_bath:
            nod = 1.0 / (np.exp(np.full((mesh.ne, 3), float(w)) / kT_phonon) - 1.0)
            b.constrain(nodal_to_linform(nod))
    if ee and electron_bands:
        for c in mat.addScatteringChannelsWildcards(["el:*"] * 4, [IN, IN, OUT, OUT], 0):
            c.amplitude = ee_amplitude
    if eph and electron_bands and phonon_energies:
        for c in mat.addScatteringChannelsWildcards(["el:*", "pn:*", "el:*"], [IN, IN, OUT], 0):
            c.amplitude = eph_amplitude
    return mat


def initial_status(mat, kT=0.1, mu=0.3, kT_phonon=0.05, seed=0, bump_amplitude=0.3, bump_sigma=0.15):
    st = MaterialStatus(mat)
    rng = np.random.default_rng(seed)
    for b in mat.bands:
        E = linform_to_nodal(b.dispersion_coeffs)
        if b.statistics == FERMION:
            fd = 1.0 / (np.exp((E - mu) / kT) + 1.0)
            cx, cy = rng.uniform(-1.0, 1.0, size=2)
            v = b.mesh.vertices()
            g = np.exp(-((v[..., 0] - cx) ** 2 + (v[..., 1] - cy) ** 2) / (2.0 * bump_sigma ** 2))
            nod = fd + bump_amplitude * (1.0 - fd) * g
        else:
            if b.constrained:
                st[b.name] = b.population_at(0.0)
                continue
            nod = 1.0 / (np.exp(E / kT_phonon) - 1.0)
        st[b.name] = nodal_to_linform(nod)
    return st


def pulsed_bath(N=6, t_pulse=0.12, width=0.02, kT_base=0.05, kT_peak=0.15, **kw):
    """Two-band e-ph + drift whose optical-phonon band (hw = 0.2, band 2) is a
    bath constrained to a Bose population at a temperature that follows a
    Gaussian pulse in time, kT(t) = kT_base + (kT_peak - kT_base)
    exp(-((t - t_pulse) / width)^2): a time-dependent constrainedPopulation,
    as a laser-heated reservoir."""
    mat = build_material(N, ("P", "D"), (0.2,), ee=False, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9,
                         phonon_bath=True, **kw)
    ph = mat.bands[2]
    ne = ph.mesh.ne

    def population(t):
        kT = kT_base + (kT_peak - kT_base) * np.exp(-((t - t_pulse) / width) ** 2)
        return nodal_to_linform(np.full((ne, 3), 1.0 / (np.exp(0.2 / kT) - 1.0)))
    ph.constrain(population)
    return mat


# The benchmark workloads, named by what they hold.
def parabolic_ee(N=16, **kw):
    """One parabolic band, e-e constant matrix element, rtol 1e-6 / atol 1e-9."""
    return build_material(N, ("P",), (), ee=True, eph=False, rtol=1e-6, atol=1e-9, **kw)


def two_band_eph_drift(N=64, ee=False, **kw):
    """Parabola + Dirac cone, optical phonon hw=0.2 (Bose kT=0.05), field (0.1,0),
    rtol 1e-8.  e-e is off by default: at N=64 its tuple lists (~1e11 per
    channel) exceed device memory; at N=32 an adjoint needs ~1200 e-e
    evaluations of ~2e9 tuples."""
    return build_material(N, ("P", "D"), (0.2,), ee=ee, eph=True, field=(0.1, 0.0), rtol=1e-8, atol=1e-9, **kw)


def three_band_two_phonon(N=128, ee=False, **kw):
    """Parabola, Dirac cone and heavy hole with two phonon branches (0.15, 0.25)."""
    return build_material(N, ("P", "D", "H"), (0.15, 0.25), ee=ee, eph=True, rtol=1e-8, atol=1e-9, **kw)


def large_batch(n_runs=16, N=128, seed=4242, **kw):
    """A batch of n_runs three-band, two-phonon runs (three_band_two_phonon,
    e-ph channels) on one N x N mesh: per run kT uniform in [0.03, 0.2], e-ph
    couplings uniform in [0.5, 2.0] and a seeded bump; one structure, so all
    runs share the tuple lists and moment tensors.  Returns (materials, initial
    state vectors)."""
    rng = np.random.default_rng(seed)
    mats, states = [], []
    for r in range(n_runs):
        kT = float(rng.uniform(0.03, 0.2))
        amp = float(rng.uniform(0.5, 2.0))
        m = three_band_two_phonon(N, eph_amplitude=amp, **kw)
        mats.append(m)
        states.append(initial_status(m, kT=kT, seed=int(rng.integers(1 << 30))).vec)
    return mats, states


def ensemble_runs(n_runs=256, seed=2024, Ns=(16, 24, 32, 48, 64), ee=False, **kw):
    """Batched ensemble: per run N uniform in Ns, kT uniform in [0.03, 0.2],
    coupling constants uniform in [0.5, 2.0] and a seeded bump; bands, phonon,
    field and tolerances as two_band_eph_drift.  All runs use the same
    Monte-Carlo seed, so runs of equal N have identical structure (shared
    tuple lists and moment tensors).  Returns (materials, initial state
    vectors)."""
    rng = np.random.default_rng(seed)
    mats, states = [], []
    for r in range(n_runs):
        N = int(rng.choice(Ns))
        kT = float(rng.uniform(0.03, 0.2))
        amp_eph = float(rng.uniform(0.5, 2.0))
        amp_ee = float(rng.uniform(0.5, 2.0))
        m = build_material(N, ("P", "D"), (0.2,), ee=ee, eph=True, field=(0.1, 0.0), rtol=1e-8, atol=1e-9,
                           eph_amplitude=amp_eph, ee_amplitude=amp_ee, **kw)
        mats.append(m)
        states.append(initial_status(m, kT=kT, seed=int(rng.integers(1 << 30))).vec)
    return mats, states
