"""Steady-state fixed-source SNAP problems (host-side input generation).

The reference builds its inputs in Snap::setup / InitMaterial / InitSource /
Snap::initialize_scattering (snap.cc:42-222, init.cc:49-191,
snap.cc:571-714).  The benchmark decks here keep the reference's geometry,
quadrature, centre material/source layout and single-chunk decomposition, but
fill the cross-section tables with the benchmark's rule (see ``make_problem``),
which replaces snap.cc:596-657.

Array layouts (shared by the CUDA path and the CPU oracle):
  cell c = (z*ny + y)*nx + x (x fastest, the reference's Fortran/SOA order,
  snap.cc:1456-1498); ``mat[c]`` int32 1-based material ids;
  ``sigt[g, m-1]``; ``slgg[g_to, m-1, g_from, l]``; ``qi[g, c]``.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Deck:
    """The subset of the SNAP input deck (snap.cc:1032-1130) on this path."""
    nx: int
    ny: int
    nz: int
    nang: int
    ng: int
    nmom: int
    epsi: float = 1e-4
    iitm: int = 5
    oitm: int = 20
    fixup: bool = True
    lx: float = 1.0
    ly: float = 1.0
    lz: float = 1.0
    sigt_perturb: float = 0.0     # per-cell +-fraction on sigma_t (adjoint deck)
    random_mix: int = 0           # edge of a central block with a 50 % material-2 mix
    seed: int = 1234
    # time dependence (timedep, tf, nsteps of the deck; snap.cc:1060-1062)
    timedep: bool = False
    tf: float = 1.0
    nsteps: int = 1
    # reference decks: material and source layouts (mat_opt 0/1/2, src_opt
    # 0/1/2/3) with the reference's own cross sections (snap.cc:571-714);
    # None: the benchmark rule of make_problem
    mat_opt: int | None = None
    src_opt: int | None = None
    # spatial chunks of the reference deck (npey, npez, ichunk); the sweep
    # covers the whole mesh as one domain (chunked and one-chunk reference
    # runs agree to rounding); they set the MMS check's per-chunk cell edges
    # and the divisor of its average
    chunks: tuple = (1, 1, 1)

    @property
    def dt(self) -> float:
        """time-step length (snap.cc:1174)"""
        return self.tf / self.nsteps

    @property
    def h(self) -> tuple:
        """hi, hj, hk as the reference derives them, 2 / (l / n)
        (snap.cc:1178-1180)"""
        return (2.0 / (self.lx / self.nx), 2.0 / (self.ly / self.ny), 2.0 / (self.lz / self.nz))

    @property
    def nmat(self) -> int:
        """materials in the cross-section tables: one for the reference's
        homogeneous layout (its material index space is [1, 1]), else two"""
        return 1 if self.mat_opt == 0 else 2

    @property
    def cmom(self) -> int:
        return self.nmom * self.nmom

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def units_per_sweep(self) -> int:
        """cell x angle x group units of one inner iteration (8 octants)."""
        return self.cells * 8 * self.nang * self.ng


# The benchmark decks.  Deck 1 is the CPU-runnable case, deck 2 the FP64
# drop-in at GPU scale, deck 3 the mixed-precision case, deck 4 the adjoint
# case, deck 5 the large forward+adjoint case.
DECKS = {
    1: Deck(16, 16, 16, nang=10, ng=4, nmom=1, epsi=1e-4, iitm=5, oitm=20),
    2: Deck(64, 64, 64, nang=36, ng=32, nmom=4, epsi=1e-6, iitm=5, oitm=50),
    3: Deck(128, 128, 128, nang=48, ng=64, nmom=4, epsi=1e-6, iitm=5, oitm=50),
    4: Deck(32, 32, 32, nang=24, ng=16, nmom=2, epsi=1e-4, iitm=5, oitm=20,
            sigt_perturb=0.1),
    5: Deck(192, 192, 192, nang=48, ng=64, nmom=3, epsi=1e-6, iitm=5, oitm=50,
            random_mix=96),
}


def deck(n: int, **overrides) -> Deck:
    return dataclasses.replace(DECKS[n], **overrides)


def central_block(n: int) -> slice:
    """0-based [n/4, 3n/4) per axis: init.cc:59-75 (i1 = n/4+1 .. i2 = 3n/4,
    1-based inclusive)."""
    return slice(n // 4, 3 * n // 4)


def sigma_t(ng: int) -> np.ndarray:
    """sigma_t[g, m-1]: 1 + 0.01 g (0-based g) in material 1, doubled in 2."""
    base = 1.0 + 0.01 * np.arange(ng, dtype=np.float64)
    return np.stack([base, 2.0 * base], axis=1)


def scattering_matrix(ng: int, nmom: int, legendre_scale: float = 0.1) -> np.ndarray:
    """slgg[g_to, m-1, g_from, l]: in-group 0.2 sigma_t, 0.3 sigma_t split
    evenly over the lower-energy (higher-index) groups, the last group keeping
    0.5 sigma_t in-group; Legendre order l scaled by legendre_scale**l."""
    st = sigma_t(ng)
    slgg = np.zeros((ng, 2, ng, nmom), dtype=np.float64)
    for m in range(2):
        for g in range(ng):
            if g == ng - 1:
                slgg[g, m, g, 0] = 0.5 * st[g, m]
            else:
                slgg[g, m, g, 0] = 0.2 * st[g, m]
                share = 0.3 * st[g, m] / (ng - 1 - g)
                for gt in range(g + 1, ng):
                    slgg[gt, m, g, 0] = share
    for l in range(1, nmom):
        slgg[..., l] = slgg[..., 0] * legendre_scale ** l
    return slgg


def reference_layout(d: Deck):
    """InitMaterial / InitSource (init.cc:49-191): material 2 in the centre
    block [n/4, 3n/4) (mat_opt 1) or the corner block [0, n/2) (mat_opt 2),
    else 1; a unit source everywhere (src_opt 0), in the centre block (1) or
    the corner block (2).  Returns mat [C] (1-based) and qi [G, C]."""
    def block(opt, n):
        if opt == 1:
            return slice(n // 4, 3 * n // 4)
        if opt == 2:
            return slice(0, n // 2)
        return slice(0, n)
    mat = np.ones((d.nz, d.ny, d.nx), dtype=np.int32)
    if d.mat_opt in (1, 2):
        mat[block(d.mat_opt, d.nz), block(d.mat_opt, d.ny), block(d.mat_opt, d.nx)] = 2
    src = np.zeros((d.nz, d.ny, d.nx))
    if d.src_opt in (0, 1, 2):
        src[block(d.src_opt, d.nz), block(d.src_opt, d.ny), block(d.src_opt, d.nx)] = 1.0
    qi = np.broadcast_to(src.reshape(1, d.cells), (d.ng, d.cells)).copy()
    return mat.reshape(d.cells), qi


def reference_cross_sections(ng: int, nmom: int, two_materials: bool):
    """Snap::initialize_scattering (snap.cc:571-714): sigma_t, sigma_a and
    sigma_s fall by 0.01 and 0.005 per group from (1, 0.5, 0.5) in material 1
    and (2, 0.8, 1.2) in material 2; slgg splits sigma_s of each source group
    into in-group, up-scatter and down-scatter shares (0.2 / 0.1 / 0.7 in
    material 1, 0.5 / 0.1 / 0.4 in material 2; the first group keeps 0.3 (0.6)
    in-group, the last 0.9), Legendre orders scaled by 0.1 then 0.5 (material
    1) or 0.8 then 0.6 (material 2).  Returns sigt [G, nmat] and
    slgg [G_to, nmat, G_from, nmom] in this package's layout."""
    nmat = 2 if two_materials else 1
    sigt = np.zeros((ng, nmat))
    sigs = np.zeros((ng, nmat))
    base = [(1.0, 0.5), (2.0, 1.2)]
    for m in range(nmat):
        sigt[0, m], sigs[0, m] = base[m]
        for g in range(1, ng):
            sigt[g, m] = 0.01 * sigt[g - 1, m]
            sigs[g, m] = 0.005 * sigs[g - 1, m]
    slgg = np.zeros((ng, nmat, ng, nmom))
    shares = [(0.2, 0.3, 0.7, 0.9), (0.5, 0.6, 0.4, 0.9)]   # in-group, first group, down, last group
    for m in range(nmat):
        if ng == 1:
            slgg[0, m, 0, 0] = sigs[0, m]
            continue
        ingroup, first, down, last = shares[m]
        for g in range(ng):                       # g: source group
            slgg[g, m, g, 0] = ingroup * sigs[g, m]
            if g > 0:
                t = 1.0 / g
                for g2 in range(g):
                    slgg[g2, m, g, 0] = 0.1 * sigs[g, m] * t
            else:
                slgg[g, m, g, 0] = first * sigs[g, m]
            if g < ng - 1:
                t = 1.0 / (ng - (g + 1))
                for g2 in range(g + 1, ng):
                    slgg[g2, m, g, 0] = down * sigs[g, m] * t
            else:
                slgg[g, m, g, 0] = last * sigs[g, m]
    scale = [(0.1, 0.5), (0.8, 0.6)]
    for m in range(nmat):
        for l in range(1, nmom):
            slgg[:, m, :, l] = (scale[m][0] if l == 1 else scale[m][1]) * slgg[:, m, :, l - 1]
    return sigt, slgg


def make_problem(d: Deck) -> dict:
    """Material map, fixed source and cross-section tables for a deck."""
    if d.mat_opt is not None:
        mat, qi = reference_layout(d)
        sigt, slgg = reference_cross_sections(d.ng, d.nmom, d.mat_opt != 0)
        return dict(mat=mat, qi=qi, sigt=sigt, slgg=slgg, nmat=sigt.shape[1])
    C = d.cells
    mat = np.ones((d.nz, d.ny, d.nx), dtype=np.int32)
    src = np.zeros((d.nz, d.ny, d.nx), dtype=np.float64)
    bz, by, bx = central_block(d.nz), central_block(d.ny), central_block(d.nx)
    if d.random_mix:
        rng = np.random.default_rng(d.seed)
        lo = [(n - d.random_mix) // 2 for n in (d.nz, d.ny, d.nx)]
        sl = tuple(slice(a, a + d.random_mix) for a in lo)
        mix = rng.random((d.random_mix,) * 3) < 0.5
        mat[sl] = np.where(mix, 2, 1)
        src[:] = np.where(mat == 1, 1.0, 0.0)   # unit source in material 1
    else:
        mat[bz, by, bx] = 2
        src[bz, by, bx] = 1.0
    qi = np.broadcast_to(src.reshape(1, C), (d.ng, C)).copy()
    sigt = sigma_t(d.ng)
    slgg = scattering_matrix(d.ng, d.nmom)
    prob = dict(mat=mat.reshape(C), qi=qi, sigt=sigt, slgg=slgg, nmat=2)
    if d.sigt_perturb:
        rng = np.random.default_rng(d.seed + 1)
        prob["sigt_scale"] = 1.0 + rng.uniform(-d.sigt_perturb, d.sigt_perturb, size=C)
    return prob


def quadrature(nang: int, nmom: int):
    """3-D quadrature and moment coefficients (snap.cc:1171-1342).

    Returns mu, eta, xi, w [nang] and ec [8, cmom, nang]; moment bands are
    stored with stride cmom = nmom**2 (the reference stores them with stride
    nmom, which overlaps octants for nmom > 1).
    """
    dm = 1.0 / nang
    mu = np.empty(nang)
    eta = np.empty(nang)
    mu[0] = 0.5 * dm
    eta[0] = 1.0 - 0.5 * dm
    for i in range(1, nang):          # same running sums as snap.cc:1208-1214
        mu[i] = mu[i - 1] + dm
        eta[i] = eta[i - 1] - dm
    xi = np.sqrt(1.0 - (mu * mu + eta * eta))
    w = np.full(nang, 0.125 / nang)
    cmom = nmom * nmom
    ec = np.zeros((8, cmom, nang))
    for oct_ in range(8):
        s_x = 1.0 if oct_ & 1 else -1.0
        s_y = 1.0 if oct_ & 2 else -1.0
        s_z = 1.0 if oct_ & 4 else -1.0
        ec[oct_, 0, :] = 1.0
        k = 1
        for l in range(1, nmom):
            for m in range(2 * l + 1):
                ec[oct_, k, :] = (s_x * mu) ** (2 * l - 1) * (s_z * xi * s_y * eta) ** m
                k += 1
    return mu, eta, xi, w, ec


def band_of(k: int) -> int:
    """Legendre band of flux moment k (band l holds moments l*l .. l*l+2l)."""
    l = 0
    while (l + 1) * (l + 1) <= k:
        l += 1
    return l
