"""Seeded synthetic inputs for the explicit update (no dataset exists for this path).

A ``BoxCase`` holds one box of the solver state in the reference layout: an
Array4-ordered float64 array of shape (NVAR, nz+2g, ny+2g, nx+2g) (component
slowest, i fastest, ghost cells filled by first-order extrapolation as the
reference's FillPatch does on non-periodic faces, Source/Vidyut.cpp:90-101), plus
the face arrays the Joule term reads: efield_ec[d] = -(phi_i - phi_{i-1})/dx_d
(MLMG's face gradient, Source/PotentialSolve.cpp:347-357) and
gradne_fc[d] = (ne_i - ne_{i-1})/dx_d.  The cell-centred field is the centred
difference of the potential (the face-to-cell average of efield_ec).

Electron temperature is stored in kelvin (Te[eV] * e/kB) and the electron energy
density is eps = 1.5 ne kB Te, as the reference initialises it
(test/models/Axisymmetric_streamer_Ar/Prob.H:80-81).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _abi as abi
from .mechanism import Mechanism, argon, synthetic, EV, K_B

BASE_SEED = 20261203


@dataclass
class BoxCase:
    mech: Mechanism
    dim: int
    n: tuple                     # cells (nx, ny, nz); nz = 1 (and ny = 1) below 3-D (2-D)
    ghost: int
    dx: tuple
    state: np.ndarray            # (NVAR, nz+2gz, ny+2gy, nx+2gx)
    efield: list                 # per direction: (1, nz, ny, nx) with +1 along d
    gradne: list
    params: dict = field(default_factory=dict)
    seed: int = BASE_SEED
    periodic: tuple = (0, 0, 0)

    @property
    def gvec(self):
        return tuple(self.ghost if d < self.dim else 0 for d in range(3))

    @property
    def lo(self):
        return (0, 0, 0)

    @property
    def hi(self):
        return tuple(self.n[d] - 1 for d in range(3))

    @property
    def ncell(self) -> int:
        return int(np.prod(self.n))

    def state_begin(self):
        g = self.gvec
        return (-g[0], -g[1], -g[2])

    def vd_params(self, **over) -> abi.VdParams:
        p = dict(self.params)
        p.update(over)
        return make_params(**p)


def make_params(dim, dx, n, dt=1e-12, Tg=300.0, Pg=101325.0, hyp_order=5, weno_scheme=3,
                precision=abi.PREC_FP64, bc=abi.BC_IHNEU, bg_mask=0, elecenergy_solve=1,
                do_reactions=1, do_transport=1, do_bg_reactions=0, floor_jh=0, const_ele_trans=0,
                cs_technique=0, bound_specden=0, ele_mob=0.0, ele_diff=0.0, min_species_density=1e10,
                min_electron_density=1e10, min_electron_temp=300.0, update_te=0, gradne_from_state=0,
                user_defined_vel=0, user_vel=(0.0, 0.0, 0.0), vel_species=0, time=0.0,
                bc_lo=None, bc_hi=None, check_finite=0) -> abi.VdParams:
    p = abi.VdParams()
    p.dim = dim
    p.hyp_order = hyp_order
    p.weno_scheme = weno_scheme
    p.user_defined_vel = user_defined_vel
    p.vel_species = vel_species
    p.precision = precision
    for d in range(3):
        p.user_vel[d] = user_vel[d]
        p.dx[d] = dx[d] if d < len(dx) else 1.0
        p.domlo[d] = 0
        p.domhi[d] = n[d] - 1
    p.Tg, p.Pg, p.time, p.dt = Tg, Pg, time, dt
    for c in range(4):
        for d in range(3):
            p.bc_lo[c][d] = (bc_lo[c][d] if bc_lo is not None else bc) if d < dim else 0
            p.bc_hi[c][d] = (bc_hi[c][d] if bc_hi is not None else bc) if d < dim else 0
    p.elecenergy_solve = elecenergy_solve
    p.do_reactions = do_reactions
    p.do_transport = do_transport
    p.do_bg_reactions = do_bg_reactions
    p.floor_jh = floor_jh
    p.const_ele_trans = const_ele_trans
    p.cs_technique = cs_technique
    p.bound_specden = bound_specden
    p.ele_mob, p.ele_diff = ele_mob, ele_diff
    p.min_species_density = min_species_density
    p.min_electron_density = min_electron_density
    p.min_electron_temp = min_electron_temp
    p.bg_mask = bg_mask
    p.update_te = update_te
    p.gradne_from_state = gradne_from_state
    p.check_finite = check_finite
    return p


# ---------------------------------------------------------------------------
def fill_ghosts(a: np.ndarray, dim: int, g: int, periodic=(0, 0, 0)) -> None:
    """foextrap (or periodic wrap) of every component, direction by direction so
    that corner ghosts are filled too.  a: (ncomp, nz+2g, ny+2g, nx+2g)."""
    for d in range(dim):
        ax = 3 - d
        n = a.shape[ax] - 2 * g
        idx = [slice(None)] * 4
        for q in range(1, g + 1):
            lo_g, hi_g = g - q, g + n - 1 + q
            if periodic[d]:
                lo_s, hi_s = g + n - 1 - ((q - 1) % n), g + ((q - 1) % n)
            else:
                lo_s, hi_s = g, g + n - 1
            idx[ax] = lo_g
            src = list(idx)
            src[ax] = lo_s
            a[tuple(idx)] = a[tuple(src)]
            idx[ax] = hi_g
            src[ax] = hi_s
            a[tuple(idx)] = a[tuple(src)]
        idx[ax] = slice(None)


def _coords(n, dx, g, dim):
    """cell-centre coordinates including ghosts, per direction."""
    out = []
    for d in range(3):
        gd = g if d < dim else 0
        out.append((np.arange(-gd, n[d] + gd) + 0.5) * dx[d])
    return out


def smooth_uniform_field(rng, n, dim: int, n_modes: int = 12, kmax: int = 2) -> np.ndarray:
    """Spatially correlated field with a uniform [0, 1) marginal: a sum of n_modes
    random cosines (at most kmax periods across the box), normalised to unit
    variance and mapped through the normal CDF.  Shape (nz, ny, nx)."""
    from math import erf, sqrt
    axes = [(np.arange(n[d]) + 0.5) / n[d] if d < dim else np.zeros(1) for d in range(3)]
    g = np.zeros((len(axes[2]), len(axes[1]), len(axes[0])))
    var = 0.0
    for _ in range(n_modes):
        k = [int(rng.integers(-kmax, kmax + 1)) if d < dim else 0 for d in range(3)]
        if not any(k):
            k[0] = 1
        a = rng.normal()
        ph = rng.uniform(0.0, 2.0 * np.pi)
        # separable evaluation: cos(A+B+C+ph) through complex exponentials
        ex = np.exp(2j * np.pi * k[0] * axes[0])
        ey = np.exp(2j * np.pi * k[1] * axes[1])
        ez = np.exp(2j * np.pi * k[2] * axes[2])
        g += a * np.real(np.exp(1j * ph) * ez[:, None, None] * ey[None, :, None] * ex[None, None, :])
        var += 0.5 * a * a
    g /= np.sqrt(max(var, 1e-30))
    try:
        from scipy.special import ndtr
        u = ndtr(g)
    except ImportError:  # pragma: no cover
        u = 0.5 * (1.0 + np.vectorize(erf, otypes=[float])(g / sqrt(2.0)))
    return np.clip(u, 0.0, 1.0 - 1e-15)


def build_case(mech: Mechanism, dim: int, n, dx, seed: int, *, density="loguniform",
               dens_range=(1e8, 1e22), blob_peak_exp=(14.0, 18.0), floor=1e10, bg_density=2.4e25,
               te_range_ev=(0.5, 5.0), voltage=1000.0, noise=0.05, ghost=3, periodic=(0, 0, 0),
               params: dict | None = None, n_modes: int = 12) -> BoxCase:
    """Seeded box: species densities (``loguniform``: independent per cell and
    species; ``loguniform_smooth``: the same log-uniform marginal but spatially
    correlated over about half the box; ``blob``: the 2-D argon config's
    Gaussian electron blob with ions matching and the other species at the
    floor), background species at ``bg_density``,
    per-cell Te uniform in te_range_ev, potential phi = V x/L (1 + noise*xi) with
    xi uniform in [-1, 1]."""
    n = tuple(int(v) for v in n) + (1,) * (3 - len(n))
    dx = tuple(float(v) for v in dx) + (1.0,) * (3 - len(dx))
    rng = np.random.default_rng(seed)
    ns = mech.ns
    g = ghost
    gv = tuple(g if d < dim else 0 for d in range(3))
    shp = (n[2] + 2 * gv[2], n[1] + 2 * gv[1], n[0] + 2 * gv[0])
    st = np.zeros((mech.nvar,) + shp, dtype=np.float64)
    inner = (slice(gv[2], gv[2] + n[2]), slice(gv[1], gv[1] + n[1]), slice(gv[0], gv[0] + n[0]))
    cshape = (n[2], n[1], n[0])
    bg = set(mech.bg_species)

    if density == "blob":
        xs = [(np.arange(n[d]) + 0.5) * dx[d] for d in range(3)]
        L = [n[d] * dx[d] for d in range(3)]
        peak = 10.0 ** rng.uniform(*blob_peak_exp)
        ctr = [L[d] * rng.uniform(0.35, 0.65) for d in range(3)]
        sig = [L[d] / 8.0 for d in range(3)]
        zz, yy, xx = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
        r2 = ((xx - ctr[0]) / sig[0]) ** 2
        if dim > 1:
            r2 = r2 + ((yy - ctr[1]) / sig[1]) ** 2
        if dim > 2:
            r2 = r2 + ((zz - ctr[2]) / sig[2]) ** 2
        ne = floor + peak * np.exp(-0.5 * r2)
        for s in range(ns):
            if s in bg:
                st[(s,) + inner] = bg_density
            elif s == mech.e_id or mech.charge[s] > 0:
                st[(s,) + inner] = ne
            else:
                st[(s,) + inner] = floor
    elif density == "loguniform_smooth":
        lo, hi = np.log10(dens_range[0]), np.log10(dens_range[1])
        for s in range(ns):
            if s in bg:
                st[(s,) + inner] = bg_density
            else:
                st[(s,) + inner] = 10.0 ** (lo + (hi - lo) * smooth_uniform_field(rng, n, dim, n_modes))
    else:
        lo, hi = np.log10(dens_range[0]), np.log10(dens_range[1])
        for s in range(ns):
            if s in bg:
                st[(s,) + inner] = bg_density
            else:
                st[(s,) + inner] = 10.0 ** rng.uniform(lo, hi, size=cshape)

    te = rng.uniform(te_range_ev[0], te_range_ev[1], size=cshape) * EV
    st[(abi.ETEMP(ns),) + inner] = te
    Lx = n[0] * dx[0]
    xc = (np.arange(n[0]) + 0.5) * dx[0]
    xi = rng.uniform(-1.0, 1.0, size=cshape)
    phi = voltage * (xc[None, None, :] / Lx) * (1.0 + noise * xi)
    st[(abi.POT(ns),) + inner] = phi
    # ghosts of the primary fields
    fill_ghosts(st, dim, g, periodic)
    # cell-centred E = -grad(phi) by centred differences (uses ghost phi)
    P = st[abi.POT(ns)]
    for d in range(3):
        comp = abi.EFX(ns) + d
        if d >= dim:
            st[comp] = 0.0
            continue
        ax = 2 - d
        sl_p = [slice(gv[2], gv[2] + n[2]), slice(gv[1], gv[1] + n[1]), slice(gv[0], gv[0] + n[0])]
        sl_m = list(sl_p)
        sl_p[ax] = slice(sl_p[ax].start + 1, sl_p[ax].stop + 1)
        sl_m[ax] = slice(sl_m[ax].start - 1, sl_m[ax].stop - 1)
        st[(comp,) + inner] = -(P[tuple(sl_p)] - P[tuple(sl_m)]) / (2.0 * dx[d])
    E2 = sum(st[abi.EFX(ns) + d][inner] ** 2 for d in range(3))
    Ntot = st[:ns][(slice(None),) + inner].sum(axis=0)
    st[(abi.REF(ns),) + inner] = np.sqrt(E2) / Ntot / 1e-21
    fill_ghosts(st, dim, g, periodic)
    # electron energy density from the (ghost-filled) ne and Te
    st[abi.EEN(ns)] = 1.5 * st[mech.e_id] * K_B * st[abi.ETEMP(ns)]

    # face arrays on the face box of the valid region
    efield, gradne = [], []
    ne_all = st[mech.e_id]
    for d in range(3):
        if d >= dim:
            efield.append(np.zeros((1, n[2], n[1], n[0])))
            gradne.append(np.zeros((1, n[2], n[1], n[0])))
            continue
        ax = 2 - d
        fn = list(cshape)
        fn[ax] += 1
        sl_r = [slice(gv[2], gv[2] + n[2]), slice(gv[1], gv[1] + n[1]), slice(gv[0], gv[0] + n[0])]
        sl_r[ax] = slice(sl_r[ax].start, sl_r[ax].stop + 1)
        sl_l = list(sl_r)
        sl_l[ax] = slice(sl_r[ax].start - 1, sl_r[ax].stop - 1)
        efield.append((-(P[tuple(sl_r)] - P[tuple(sl_l)]) / dx[d]).reshape((1,) + tuple(fn)))
        gradne.append(((ne_all[tuple(sl_r)] - ne_all[tuple(sl_l)]) / dx[d]).reshape((1,) + tuple(fn)))

    prm = dict(dim=dim, dx=dx, n=n, bg_mask=mech.bg_mask())
    if params:
        prm.update(params)
    return BoxCase(mech=mech, dim=dim, n=n, ghost=g, dx=dx, state=np.ascontiguousarray(st),
                   efield=[np.ascontiguousarray(e) for e in efield],
                   gradne=[np.ascontiguousarray(e) for e in gradne], params=prm, seed=seed,
                   periodic=periodic)


# ---------------------------------------------------------------------------
# The configurations of the workload.  Each returns a BoxCase (or a list of them).
def config_argon2d(seed: int = BASE_SEED, n=(256, 256), n_reactions: int = 10) -> BoxCase:
    """2-D single box, dx = 1e-5 m; E, Ar+, Ar*, constant Ar background 2.4e25;
    Gaussian electron blob peaking at 10^U(14,18) over a 1e10 floor with Ar+ = ne
    and Ar* at the floor; 0-1 kV ramp with 5 % noise; Te uniform 0.5-5 eV; ten
    Arrhenius reactions; one explicit step, dt = 1e-12 s."""
    mech = argon(n_reactions, seed + 1)
    return build_case(mech, 2, n, (1e-5, 1e-5), seed + 2, density="blob", te_range_ev=(0.5, 5.0),
                      voltage=1000.0, params=dict(dt=1e-12))


def config_precision3d(seed: int = BASE_SEED, n=(128, 128, 128), n_species: int = 24,
                       n_reactions: int = 150) -> BoxCase:
    """3-D single box: 24 species / 150 reactions, densities log-uniform 1e8-1e22
    (spatially correlated; background gas 2.4e25), Te 0.3-10 eV per cell,
    potential ramp + noise; one step."""
    mech = synthetic(n_species, n_reactions, seed + 11)
    return build_case(mech, 3, n, (1e-5, 1e-5, 1e-5), seed + 12, density="loguniform_smooth",
                      dens_range=(1e8, 1e22), te_range_ev=(0.3, 10.0), voltage=1000.0,
                      params=dict(dt=1e-12))


def face_gradients(case: BoxCase, state: np.ndarray) -> list:
    """gradne_fc[d] = (ne_i - ne_{i-1}) / dx_d on the face box of direction d, from
    the electron density of `state` (laid out like case.state)."""
    g = case.gvec
    n = case.n
    ne = state[case.mech.e_id]
    out = []
    for d in range(3):
        if d >= case.dim:
            out.append(np.zeros((1, n[2], n[1], n[0])))
            continue
        ax = 2 - d
        fn = [n[2], n[1], n[0]]
        fn[ax] += 1
        sl_r = [slice(g[2], g[2] + n[2]), slice(g[1], g[1] + n[1]), slice(g[0], g[0] + n[0])]
        sl_r[ax] = slice(sl_r[ax].start, sl_r[ax].stop + 1)
        sl_l = list(sl_r)
        sl_l[ax] = slice(sl_r[ax].start - 1, sl_r[ax].stop - 1)
        out.append(np.ascontiguousarray(((ne[tuple(sl_r)] - ne[tuple(sl_l)]) / case.dx[d]).reshape((1,) + tuple(fn))))
    return out


# parameters of a case that takes many steps: the state evolves, so the Joule
# term's density gradient is taken from it, Te follows the energy, and densities
# are clipped at the floors as the species solve does
MULTISTEP_PARAMS = dict(dt=1e-12, gradne_from_state=1, update_te=1, bound_specden=1)


def config_batched(seed: int = BASE_SEED, n_cases: int = 64, side=(64, 512), n_species: int = 8,
                   n_reactions: int = 40, dens_range=(1e10, 1e18)):
    """Batched workload: n_cases independent 2-D cases, each side length drawn
    log-uniform in `side` (uneven boxes), one shared 8-species / 40-reaction
    synthetic mechanism, densities log-uniform (spatially correlated) in
    dens_range, Te 0.3-10 eV, 1 kV ramp + 5 % noise, dx = 1e-5 m.  Returns
    (mechanism, [BoxCase])."""
    mech = synthetic(n_species, n_reactions, seed + 21)
    rng = np.random.default_rng(seed + 22)
    lo, hi = np.log(side[0]), np.log(side[1])
    cases = []
    for i in range(n_cases):
        nx = int(round(float(np.exp(rng.uniform(lo, hi)))))
        ny = int(round(float(np.exp(rng.uniform(lo, hi)))))
        cases.append(build_case(mech, 2, (nx, ny), (1e-5, 1e-5), seed + 1000 + i, density="loguniform_smooth",
                                dens_range=dens_range, te_range_ev=(0.3, 10.0), voltage=1000.0,
                                params=dict(MULTISTEP_PARAMS)))
    return mech, cases


SERVING_ADVECTIVE_CFL = 0.2
SERVING_DT_MAX = 2e-13


def electron_time_scales(case: BoxCase) -> tuple:
    """(dt_edrift, dt_diel_relax) of the case's initial state as
    Vidyut::find_time_scales computes them (Source/TimeStep.cpp:32-118):
    min over directions of dx / max |mu_e| |E|, and eps0 / (e max |mu_e| ne), for
    the collisional electron mobility (VD_MOB_ELECTRON) of the synthetic
    mechanisms."""
    m = case.mech
    if m.mob_kind[m.e_id] != abi.MOB_ELECTRON:
        raise NotImplementedError("time scales of this electron mobility model")
    ns, g = m.ns, case.gvec
    v = (slice(g[2], g[2] + case.n[2]), slice(g[1], g[1] + case.n[1]), slice(g[0], g[0] + case.n[0]))
    st = case.state
    N = st[:ns][(slice(None),) + v].sum(axis=0)
    te = st[abi.ETEMP(ns)][v]
    emag = np.sqrt(sum(st[abi.EFX(ns) + d][v] ** 2 for d in range(3)))
    echarge, me, eps0 = 1.60217662e-19, 9.10938188e-31, 8.854187817e-12
    mu = (echarge / me) / (np.sqrt(8.0 * K_B * te / np.pi / me) * N * m.mob_p0[m.e_id])
    dt_edrift = min(case.dx[:case.dim]) / float((mu * emag).max())
    dt_diel = eps0 / echarge / float((mu * st[m.e_id][v]).max())
    return dt_edrift, dt_diel


def config_serving(seed: int = BASE_SEED, n_requests: int = 48, rate_per_s: float = 500.0,
                   side=(256, 1024), steps=(50, 2000), voltage_kv=(0.5, 5.0), pressure_bar=(0.1, 10.0),
                   frac_2d: float = 0.5):
    """Serving workload: a Poisson request stream at rate_per_s of 1-D and 2-D
    discharge cases (2-D with probability frac_2d).  Each case: sides log-uniform
    in `side` cells, applied voltage uniform in voltage_kv (the potential ramp's
    amplitude), pressure log-uniform in pressure_bar scaling the background gas
    (2.4e25 m^-3 at 1 bar), step count log-uniform in `steps`, the batched
    workload's 8-species / 40-reaction mechanism.  Each case's time step is the
    reference's adaptive one for its initial state (Source/TimeStep.cpp:14-31:
    the electron drift and dielectric relaxation limits times their CFL numbers,
    capped at dt_max), with an advective CFL of SERVING_ADVECTIVE_CFL and
    dt_max = SERVING_DT_MAX: the explicit forward-Euler update needs both smaller
    than the reference's semi-implicit defaults (CFL 0.7).  At dt = 1e-12 s most
    requests of this distribution (fields up to ~2e7 V/m at 0.1-10 bar, up to 2000
    steps) heat their electrons without bound and overflow, in the CPU oracle as
    on the GPU; at 2e-13 s the 1-D ones checked with the oracle stay finite.
    Returns (mechanism, [(arrival time [s], BoxCase, nsteps)])."""
    mech = synthetic(8, 40, seed + 21)
    rng = np.random.default_rng(seed + 31)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += float(rng.exponential(1.0 / rate_per_s))
        dim = 2 if rng.uniform() < frac_2d else 1
        n = tuple(int(round(float(np.exp(rng.uniform(np.log(side[0]), np.log(side[1])))))) for _ in range(dim))
        v = float(rng.uniform(*voltage_kv)) * 1e3
        p = float(np.exp(rng.uniform(np.log(pressure_bar[0]), np.log(pressure_bar[1]))))
        ns = int(round(float(np.exp(rng.uniform(np.log(steps[0]), np.log(steps[1]))))))
        case = build_case(mech, dim, n, (1e-5,) * dim, seed + 5000 + i, density="loguniform_smooth",
                          dens_range=(1e10, 1e18), te_range_ev=(0.3, 10.0), voltage=v, bg_density=2.4e25 * p,
                          params=dict(MULTISTEP_PARAMS), n_modes=4)
        dt_edrift, dt_diel = electron_time_scales(case)
        case.params["dt"] = min(SERVING_DT_MAX, SERVING_ADVECTIVE_CFL * dt_edrift, dt_diel)
        out.append((t, case, ns))
    return mech, out


def config_large_device(device="cuda", seed: int = BASE_SEED, n=(384, 384, 384), n_species: int = 12,
                        n_reactions: int = 60, dens_range=(1e10, 1e18), te_range_ev=(0.3, 10.0),
                        voltage: float = 1000.0, n_modes: int = 4, ghost: int = 3):
    """Large single case, built on the GPU (a 384^3 state is 10 GB; numpy would take
    minutes): 3-D box, synthetic 12-species / 60-reaction mechanism, every
    non-background species log-uniform in dens_range and spatially correlated (a
    sum of n_modes random cosines mapped through the normal CDF, as
    smooth_uniform_field), background gas 2.4e25, Te uniform in te_range_ev per
    cell, potential initialised to the ramp V (1 - x/L) (the potential step
    replaces it), dx = 1e-5 m.  Returns (mechanism, BoxCase without host arrays,
    device state tensor of shape (NVAR, nz+2g, ny+2g, nx+2g))."""
    import torch
    mech = synthetic(n_species, n_reactions, seed + 31)
    gen = torch.Generator(device="cpu").manual_seed(seed + 32)
    ns = mech.ns
    dim = 3
    n = tuple(int(v) for v in n)
    shp = (mech.nvar, n[2] + 2 * ghost, n[1] + 2 * ghost, n[0] + 2 * ghost)
    st = torch.zeros(shp, dtype=torch.float64, device=device)
    inner = (slice(ghost, ghost + n[2]), slice(ghost, ghost + n[1]), slice(ghost, ghost + n[0]))
    axes = [(torch.arange(n[d], device=device, dtype=torch.float64) + 0.5) / n[d] for d in range(3)]
    lo, hi = np.log10(dens_range[0]), np.log10(dens_range[1])
    bg = set(mech.bg_species)
    for s in range(ns):
        if s in bg:
            st[(s,) + inner] = 2.4e25
            continue
        g = torch.zeros((n[2], n[1], n[0]), dtype=torch.float64, device=device)
        var = 0.0
        for _ in range(n_modes):
            k = [int(torch.randint(-2, 3, (1,), generator=gen)) for _ in range(3)]
            if not any(k):
                k[0] = 1
            a = float(torch.randn(1, generator=gen))
            ph = float(torch.rand(1, generator=gen)) * 2.0 * np.pi
            cz = torch.cos(2 * np.pi * k[2] * axes[2])[:, None, None]
            sz = torch.sin(2 * np.pi * k[2] * axes[2])[:, None, None]
            xy = 2 * np.pi * (k[0] * axes[0][None, None, :] + k[1] * axes[1][None, :, None]) + ph
            g += a * (torch.cos(xy) * cz - torch.sin(xy) * sz)  # cos(xy + z)
            var += 0.5 * a * a
        g /= max(var, 1e-30) ** 0.5
        u = torch.special.ndtr(g).clamp(0.0, 1.0 - 1e-15)
        st[(s,) + inner] = torch.pow(10.0, lo + (hi - lo) * u)
        del g, u
    te = torch.rand((n[2], n[1], n[0]), generator=gen, dtype=torch.float64).to(device)
    st[(abi.ETEMP(ns),) + inner] = (te_range_ev[0] + (te_range_ev[1] - te_range_ev[0]) * te) * EV
    del te
    x = (torch.arange(n[0], device=device, dtype=torch.float64) + 0.5) / n[0]
    st[(abi.POT(ns),) + inner] = (voltage * (1.0 - x))[None, None, :]
    # ghosts by first-order extrapolation, then the energy density from ne and Te
    for d in range(3):
        ax = 3 - d
        for q in range(1, ghost + 1):
            lo_idx = [slice(None)] * 4
            src = [slice(None)] * 4
            lo_idx[ax] = ghost - q
            src[ax] = ghost
            st[tuple(lo_idx)] = st[tuple(src)]
            lo_idx[ax] = ghost + n[d] - 1 + q
            src[ax] = ghost + n[d] - 1
            st[tuple(lo_idx)] = st[tuple(src)]
    st[abi.EEN(ns)] = 1.5 * st[mech.e_id] * K_B * st[abi.ETEMP(ns)]
    prm = dict(dim=dim, dx=(1e-5,) * 3, n=n, bg_mask=mech.bg_mask(), **MULTISTEP_PARAMS)
    case = BoxCase(mech=mech, dim=dim, n=n, ghost=ghost, dx=(1e-5,) * 3, state=None, efield=[], gradne=[],
                   params=prm, seed=seed)
    return mech, case, st
