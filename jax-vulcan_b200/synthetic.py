"""Seeded synthetic workloads for the Ros2 step (no public dataset exists).

Every workload is generated from a ``numpy.random.default_rng`` seed:

* a random element-balanced mass-action network, written in the network-file
  format and parsed back (`network.py`);
* an atmosphere: log-spaced pressure, a smooth monotone T(z), log-uniform Kzz,
  log-uniform mixing ratios normalised to ``n = P / (k_B T)``, and the
  hydrostatic geometry of reference `atm_setup.py:23-38` (interface pressures)
  and `atm_setup.py:253-375` (g, Hp, dz, dzi, Ti, Hpi);
* log-uniform rate constants ``k[nr+1, nz]`` (row 0 is the unused slot).

The named configurations mirror the five benchmark configurations of the
Ros2 step: ``config0`` (one atmosphere, ni=69, 700+700 reactions, nz=120),
``config1`` (config0 plus 40 photolysis branches over 2500 wavelength bins),
``config2`` (256 uneven atmospheres), ``config3`` (SNCHO-shaped ni=89,
nr=2000, nz=150, stiff k) and ``config4`` (adjoint shapes).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .network import NetworkTables, format_network, parse_network_text

# CGS constants (reference `phy_const.py:1-9`).
KB = 1.38064852e-16
NAVO = 6.02214086e23
HC = 1.98644582e-9

ATOM_MASS = {"C": 12.011, "H": 1.008, "O": 15.999, "N": 14.007, "S": 32.06}

# HD 189733b planet constants used for the geometry (reference `vulcan_cfg.py:43,68,70,81`).
GS = 2140.0
RP = 1.138 * 7.1492e9
P_B = 1e9


@dataclass
class SyntheticNetwork:
    text: str
    tables: NetworkTables
    elements: tuple
    compo: np.ndarray          # [ni, n_elements] atom counts, in parsed species order
    ms: np.ndarray             # [ni] molar masses (g/mol)
    photo_branches: list = field(default_factory=list)   # [(species, branch, row)]


def _rng(seed, *tags):
    """Generator seeded from an int or a tuple of ints plus stream tags."""
    return np.random.default_rng([int(x) for x in np.atleast_1d(seed)] + list(tags))


def _species_set(rng, ni, elements):
    ne = len(elements)
    seen = set()
    vecs = []
    while len(vecs) < ni:
        v = tuple(int(x) for x in rng.integers(0, 5, size=ne))
        if sum(v) == 0 or v in seen:
            continue
        seen.add(v)
        vecs.append(v)
    return np.array(vecs, dtype=np.int64)


def _name(v, elements):
    return "".join(f"{e}{c if c > 1 else ''}" for e, c in zip(elements, v) if c > 0)


def _balanced_reactions(rng, V, n_fwd):
    """Draw ``n_fwd`` element-balanced reactions (1-2 reactants, 1-3 products).

    Every reactant multiset with at least one balanced product multiset is
    enumerated first; draws then favour reactions that touch a species not yet
    used, so every species appears in the network.
    """
    ni = V.shape[0]
    singles: dict = {}
    pairs: dict = {}
    for i in range(ni):
        singles.setdefault(tuple(V[i]), []).append((i,))
        for j in range(i, ni):
            pairs.setdefault(tuple(V[i] + V[j]), []).append((i, j))
    options = []
    for reac in [(i,) for i in range(ni)] + [(i, j) for i in range(ni) for j in range(i, ni)]:
        tot = V[list(reac)].sum(axis=0)
        cands = list(singles.get(tuple(tot), [])) + list(pairs.get(tuple(tot), []))
        for p in range(ni):
            rem = tot - V[p]
            if (rem < 0).any():
                continue
            cands += [(p, a, b) for (a, b) in pairs.get(tuple(rem), []) if p <= a]
        cands = [c for c in cands if sorted(c) != sorted(reac)]
        if cands:
            options.append((reac, cands))
    if not options:
        raise RuntimeError("no balanced reaction exists for this species set")
    used = np.zeros(ni, dtype=bool)
    out = []
    for _ in range(n_fwd):
        pick = None
        if not used.all():
            fresh = [o for o in options
                     if (~used[list(o[0])]).any() or any((~used[list(c)]).any() for c in o[1])]
            if fresh:
                pick = fresh[int(rng.integers(0, len(fresh)))]
        if pick is None:
            pick = options[int(rng.integers(0, len(options)))]
        reac, cands = pick
        if not used.all():
            new = [c for c in cands if (~used[list(c)]).any()]
            cands = new or cands
        prod = cands[int(rng.integers(0, len(cands)))]
        reac = list(reac)
        if len(reac) == 2 and rng.random() < 0.5:
            reac = reac[::-1]
        prod = [prod[i] for i in rng.permutation(len(prod))]
        out.append((reac, prod))
        used[reac] = True
        used[prod] = True
    return out, used


def _side(idx, names):
    acc: dict = {}
    for i in idx:
        acc[names[i]] = acc.get(names[i], 0) + 1
    return [(c, s) for s, c in acc.items()]


def make_network(seed: int, ni: int, n_fwd: int, elements=("C", "H", "O", "N"),
                 n_photo: int = 0, n_three_body: int = 0) -> SyntheticNetwork:
    """Random element-balanced network with every species used.

    ``n_photo`` photolysis branches (1 reactant, 2-3 balanced products) are
    written in a ``# photo`` section after ``# reverse stops``; the last
    ``n_three_body`` reactions go to the three-body section (``+ M``).
    """
    for attempt in range(64):
        rng = _rng(seed, attempt)
        V = _species_set(rng, ni, elements)
        try:
            rxns, used = _balanced_reactions(rng, V, n_fwd)
        except RuntimeError:
            continue
        if not used.all():
            continue
        names = [_name(v, elements) for v in V]
        photo = []
        if n_photo:
            pairs: dict = {}
            for i in range(ni):
                for j in range(i, ni):
                    pairs.setdefault(tuple(V[i] + V[j]), []).append((i, j))
            branch_count: dict = {}
            order = rng.permutation(ni)
            guard = 0
            while len(photo) < n_photo and guard < 100000:
                guard += 1
                sp = int(order[guard % ni])
                cands = [c for c in pairs.get(tuple(V[sp]), []) if sp not in c]
                if not cands:
                    continue
                prod = list(cands[int(rng.integers(0, len(cands)))])
                br = branch_count.get(sp, 0) + 1
                if br > 3:
                    continue
                branch_count[sp] = br
                photo.append((names[sp], br, _side(prod, names)))
            if len(photo) < n_photo:
                continue
        sides = [(_side(r, names), _side(p, names)) for r, p in rxns]
        n2 = len(sides) - n_three_body
        text = format_network(sides[:n2], three_body=sides[n2:], photo=photo)
        tables = parse_network_text(text)
        if tables.ni != ni:
            continue
        pos = {s: k for k, s in enumerate(names)}
        perm = np.array([pos[s] for s in tables.species])
        compo = V[perm].astype(np.float64)
        ms = compo @ np.array([ATOM_MASS[e] for e in elements])
        branches = [(sp, br, tables.pho_rate_index[(sp, br)]) for sp, br, _ in photo]
        return SyntheticNetwork(text=text, tables=tables, elements=tuple(elements),
                                compo=compo, ms=ms, photo_branches=branches)
    raise RuntimeError("no balanced network found for this seed")


def compute_pico(pco):
    """Interface pressures from cell centres (reference `atm_setup.py:23-38`)."""
    pco = np.asarray(pco, dtype=np.float64)
    inner = np.sqrt(pco[1:] * pco[:-1])
    bottom = pco[0] ** 1.5 * pco[1] ** -0.5
    top = pco[-1] ** 1.5 * pco[-2] ** -0.5
    return np.concatenate([[bottom], inner, [top]])


def hydrostatic_geometry(Tco, mu, pico, gs=GS, rp=RP, p_b=P_B):
    """g, Hp, dz, dzi, zco, Ti, Hpi by the height integration of reference
    `atm_setup.py:253-375` (gas giant anchored at the 1-bar interface)."""
    nz = Tco.shape[0]
    if p_b >= 1e6:
        pref = int(np.argmin(np.abs(np.log10(pico) - 6.0)))
    else:
        pref = 0
    pref = min(pref, nz - 1)
    g = np.zeros(nz)
    Hp = np.zeros(nz)
    dz = np.zeros(nz)
    zco = np.zeros(nz + 1)
    z = 0.0
    for k, i in enumerate(range(pref, nz)):
        gi = gs if k == 0 else gs * (rp / (rp + z)) ** 2
        Hp[i] = KB * Tco[i] / (mu[i] / NAVO * gi)
        g[i] = gi
        dz[i] = Hp[i] * np.log(pico[i] / pico[i + 1])
        z = z + dz[i]
        zco[i + 1] = z
    z = 0.0
    for i in range(pref - 1, -1, -1):
        gi = gs * (rp / (rp + z)) ** 2
        Hp[i] = KB * Tco[i] / (mu[i] / NAVO * gi)
        g[i] = gi
        dz[i] = Hp[i] * np.log(pico[i] / pico[i + 1])
        z = z - dz[i]
        zco[i] = z
    dzi = 0.5 * (dz[1:] + dz[:-1])
    Ti = 0.5 * (Tco[1:] + Tco[:-1])
    Hpi = 0.5 * (Hp[1:] + Hp[:-1])
    return dict(g=g, Hp=Hp, dz=dz, dzi=dzi, zco=zco, Ti=Ti, Hpi=Hpi)


def make_atmosphere(seed, net: SyntheticNetwork, nz=120, T_offset=0.0, kzz_scale=1.0,
                    ymix_floor=1e-20, moldiff=False, advection=False, fluxes=False):
    """Seeded atmosphere for one network. Returns a dict of float64 arrays with
    the AtmStatic fields (reference `jax_step.py:26-49`) plus y, ymix, n, pco,
    Tco, dz, bins-independent geometry.

    ``moldiff``/``advection``/``fluxes`` switch on the optional transport terms
    (molecular diffusion with thermal diffusion, vertical/molecular advection
    and settling, boundary fluxes and deposition) with seeded magnitudes, so the
    parity tests exercise every branch of the diffusion assembly.
    """
    rng = _rng(seed, 7)
    ni = net.tables.ni
    pco = np.logspace(np.log10(1e2 * 1e6), np.log10(1e-8 * 1e6), nz)
    x = np.linspace(0.0, 1.0, nz)
    Tco = 800.0 + 1200.0 * (1.0 - 0.5 * (1.0 + np.tanh(4.0 * (x - 0.45)))) + T_offset
    Tco = np.maximum(Tco, 100.0)
    Kzz = 10.0 ** rng.uniform(7.0, 10.0, nz - 1) * kzz_scale
    lo = np.log10(ymix_floor)
    ymix = 10.0 ** rng.uniform(lo, 0.0, (nz, ni))
    ymix /= ymix.sum(axis=1, keepdims=True)
    n = pco / (KB * Tco)
    y = ymix * n[:, None]
    mu = ymix @ net.ms
    pico = compute_pico(pco)
    geo = hydrostatic_geometry(Tco, mu, pico)
    atm = dict(
        Kzz=Kzz,
        Dzz=np.zeros((nz - 1, ni)),
        dzi=geo["dzi"],
        vz=np.zeros(nz - 1),
        Hpi=geo["Hpi"],
        Ti=geo["Ti"],
        Tco=Tco,
        g=geo["g"],
        ms=net.ms.copy(),
        alpha=np.zeros(ni),
        M=n.copy(),
        vm=np.zeros((nz, ni)),
        vs=np.zeros((nz - 1, ni)),
        top_flux=np.zeros(ni),
        bot_flux=np.zeros(ni),
        bot_vdep=np.zeros(ni),
        gas_indx_mask=np.ones(ni, dtype=bool),
        use_vm_mol=False,
        use_settling=False,
        use_topflux=False,
        use_botflux=False,
    )
    if moldiff:
        atm["Dzz"] = 10.0 ** rng.uniform(3.0, 8.0, (nz - 1, ni))
        atm["alpha"] = rng.uniform(-0.5, 0.5, ni)
    if advection:
        atm["vz"] = rng.normal(0.0, 1.0, nz - 1)
        atm["vm"] = rng.normal(0.0, 0.3, (nz, ni))
        atm["vs"] = rng.normal(0.0, 0.1, (nz - 1, ni))
        atm["use_vm_mol"] = True
        atm["use_settling"] = True
        atm["gas_indx_mask"] = rng.random(ni) > 0.1
        atm["gas_indx_mask"][0] = True
    if fluxes:
        atm["top_flux"] = rng.normal(0.0, 1e6, ni)
        atm["bot_flux"] = 10.0 ** rng.uniform(4.0, 8.0, ni)
        atm["bot_vdep"] = 10.0 ** rng.uniform(-3.0, 0.0, ni)
        atm["use_topflux"] = True
        atm["use_botflux"] = True
    extra = dict(y=y, ymix=ymix, n=n, pco=pco, pico=pico, dz=geo["dz"], zco=geo["zco"],
                 mu=mu, Hp=geo["Hp"])
    return atm, extra


def make_rates(seed, net: SyntheticNetwork, nz, lo=-40.0, hi=-8.0, n_ref=None):
    """Log-uniform rate constants ``k[nr+1, nz]`` with row 0 (unused) zero.

    With ``n_ref`` set, each reaction's draw is divided by
    ``n_ref**(order-1)`` (order = summed reactant stoichiometry, plus one for a
    three-body reaction whose rate is multiplied by M), so the
    pseudo-first-order rate ``k * n**(order-1)`` is log-uniform in
    ``[10**lo, 10**hi]`` whatever the molecularity: the "mild" chemistry used
    for well-conditioned parity cases.
    """
    rng = _rng(seed, 11)
    nr = net.tables.nr
    k = 10.0 ** rng.uniform(lo, hi, (nr + 1, nz))
    if n_ref is not None:
        order = net.tables.reactant_stoich.sum(axis=1) + net.tables.is_three_body
        k = k / float(n_ref) ** np.maximum(order - 1.0, 0.0)[:, None]
    k[0] = 0.0
    k[net.tables.is_photo] = 0.0
    return k


@dataclass
class StepCase:
    """One seeded Ros2-step input: network, atmosphere, state, rates, dt."""
    net: SyntheticNetwork
    atm: dict
    extra: dict
    y: np.ndarray
    k: np.ndarray
    dt: float


def make_case(seed=0, ni=69, n_fwd=700, nz=120, dt=1e-6, elements=("C", "H", "O", "N"),
              k_range=(-40.0, -8.0), net=None, n_three_body=0, n_photo=0, mild=False,
              **atm_kw) -> StepCase:
    """A complete single-atmosphere step input (config 0 at the defaults).

    ``mild=True`` draws order-scaled rate constants (see `make_rates`) with
    ``k_range`` as the pseudo-first-order range: a well-conditioned step.
    """
    if net is None:
        net = make_network(seed, ni, n_fwd, elements, n_photo=n_photo, n_three_body=n_three_body)
    atm, extra = make_atmosphere(seed, net, nz=nz, **atm_kw)
    n_ref = float(np.max(extra["n"])) if mild else None
    k = make_rates(seed, net, nz, *k_range, n_ref=n_ref)
    return StepCase(net=net, atm=atm, extra=extra, y=extra["y"].copy(), k=k, dt=float(dt))


def config0(seed=0) -> StepCase:
    """Plain FP64 step: ni=69 C/H/O/N, 700+700 reactions, nz=120, dt=1e-6."""
    return make_case(seed=seed)


def config3_case(seed=3, net=None) -> StepCase:
    """SNCHO-shaped stiff case: ni=89, nr=2000, nz=150, k in [1e-45, 1e-6]."""
    return make_case(seed=seed, ni=89, n_fwd=1000, nz=150,
                     elements=("C", "H", "O", "N", "S"), k_range=(-45.0, -6.0), net=net)


def config2_batch(seed=2, batch=256):
    """Uneven batch: nz ~ U[60,200], ni in {30, 69, 89} (370/1400/2000 reactions),
    T offset +-300 K, Kzz x[0.1,10], dt log-uniform in [1e-8, 1e-2]."""
    rng = _rng(seed, 2)
    nets = {30: make_network(seed + 100, 30, 185),
            69: make_network(seed + 101, 69, 700),
            89: make_network(seed + 102, 89, 1000, elements=("C", "H", "O", "N", "S"))}
    cases = []
    for b in range(batch):
        ni = int(rng.choice([30, 69, 89]))
        nz = int(rng.integers(60, 201))
        net = nets[ni]
        atm, extra = make_atmosphere([seed, b], net, nz=nz,
                                     T_offset=float(rng.uniform(-300, 300)),
                                     kzz_scale=float(10.0 ** rng.uniform(-1, 1)))
        k = make_rates([seed, b], net, nz)
        dt = float(10.0 ** rng.uniform(-8, -2))
        cases.append(StepCase(net=net, atm=atm, extra=extra, y=extra["y"].copy(), k=k, dt=dt))
    return nets, cases


def make_bins(bin_min=2.0, bin_max=802.0, dbin1=0.125, dbin2=0.5, trans=152.0):
    """Two-resolution wavelength grid (reference `photo_setup.py:124-139`).

    The defaults give exactly 2500 bins between 2 and 801.5 nm (1200 fine bins
    below 152 nm, 1300 coarse bins above); every value is exact in binary.
    """
    if bin_min <= trans <= bin_max:
        bins = np.concatenate((np.arange(bin_min, trans, dbin1), np.arange(trans, bin_max, dbin2)))
    else:
        bins = np.arange(bin_min, bin_max, dbin1)
    din12 = int(np.flatnonzero(bins == trans)[0]) if (bins == trans).any() else len(bins)
    return bins, din12


def make_photo(seed, net: SyntheticNetwork, Tco, bins, din12, dbin1=0.125, dbin2=0.5,
               n_T_abs=4, n_scat=2):
    """Seeded photochemistry inputs for one atmosphere.

    Absorbers are the photolysing species; cross sections are smooth positive
    log-normal bumps clipped to [1e-24, 1e-17] cm^2; ``n_T_abs`` of them carry
    a linear temperature dependence (per-layer cross sections, reference
    `photo.py:15-32`). The two most abundant-by-index bulk species scatter with
    a Rayleigh lambda^-4 law. Branch cross sections are the parent's absorption
    times a seeded branching ratio; branches of T-dependent parents use the
    per-layer table (`PhotoJData`, reference `photo.py:248-266`). The stellar
    flux is a 5800 K blackbody with log-normal line jitter.
    """
    rng = _rng(seed, 13)
    t = net.tables
    nbin = bins.shape[0]
    nz = Tco.shape[0]
    sp_names = list(t.species)
    photo_sp = list(t.photo_sp)
    lam = bins

    def smooth_cross(n):
        out = np.zeros((n, nbin))
        for s in range(n):
            c = rng.uniform(np.log(20.0), np.log(400.0), 3)
            w = rng.uniform(0.2, 0.8, 3)
            amp = rng.uniform(-24.0, -17.0, 3)
            ll = np.log(lam)[None, :]
            logs = np.log10(np.sum(10.0 ** amp[:, None] * np.exp(-0.5 * ((ll - c[:, None]) / w[:, None]) ** 2), axis=0) + 1e-30)
            out[s] = 10.0 ** np.clip(logs, -24.0, -17.0)
        return out

    base = smooth_cross(len(photo_sp))
    T_sp = photo_sp[:n_T_abs]
    nonT_sp = photo_sp[n_T_abs:]
    slope = rng.uniform(-0.5, 0.5, len(T_sp))
    Tfac = 1.0 + slope[:, None] * (Tco[None, :] - 1000.0) / 1000.0       # [nT, nz]
    absp_T_cross = base[:len(T_sp)][:, None, :] * Tfac[:, :, None]
    absp_cross = base[len(T_sp):]
    scat_sp = [sp for sp in sp_names if sp not in photo_sp][:n_scat]
    scat_cross = np.stack([8.0e-24 * (500.0 / lam) ** 4 * rng.uniform(0.5, 2.0) for _ in scat_sp]) \
        if scat_sp else np.zeros((0, nbin))
    # branches: (species, branch, k row)
    br_nonT, br_T = [], []
    cross_J, cross_J_T = [], []
    for sp, br, row in net.photo_branches:
        ratio = rng.uniform(0.1, 1.0)
        if sp in T_sp:
            br_T.append((sp, br, row))
            cross_J_T.append(absp_T_cross[T_sp.index(sp)] * ratio)
        else:
            br_nonT.append((sp, br, row))
            cross_J.append(absp_cross[nonT_sp.index(sp)] * ratio)
    cross_J = np.array(cross_J).reshape(len(br_nonT), nbin)
    cross_J_T = np.array(cross_J_T).reshape(len(br_T), nz, nbin)
    hc = HC
    h, c, kb = 6.62607015e-27, 2.99792458e10, KB
    lam_cm = lam * 1e-7
    Bl = 2 * h * c ** 2 / lam_cm ** 5 / (np.exp(np.minimum(h * c / (lam_cm * kb * 5800.0), 700.0)) - 1.0)
    geom = (0.805 * 6.957e10 / (1.49597871e13 * 0.03142)) ** 2
    sflux_top = np.pi * Bl * 1e-7 * geom * np.exp(rng.normal(0.0, 0.3, nbin))
    return dict(
        absp_idx=np.array([sp_names.index(s) for s in nonT_sp], dtype=np.int64),
        absp_cross=absp_cross,
        absp_T_idx=np.array([sp_names.index(s) for s in T_sp], dtype=np.int64),
        absp_T_cross=absp_T_cross,
        scat_idx=np.array([sp_names.index(s) for s in scat_sp], dtype=np.int64),
        scat_cross=scat_cross,
        cross_J=cross_J, cross_J_T=cross_J_T,
        branch_re_idx=np.array([r for _, _, r in br_nonT], dtype=np.int64),
        branch_T_re_idx=np.array([r for _, _, r in br_T], dtype=np.int64),
        din12_indx=int(din12), dbin1=float(dbin1), dbin2=float(dbin2),
        bins=bins, sflux_top=sflux_top, mu_zenith=float(np.cos(48.0 / 180.0 * 3.14159)),
        edd=0.5, ag0=0.0, hc=hc, f_diurnal=1.0,
    )


def _eq_of(tables, row):
    """Reaction text of a parsed row (reactants -> products, M restored)."""
    sp = tables.species

    def side(idx, st, m):
        terms = [(sp[i] if s == 1 else f"{int(s)}*{sp[i]}") for i, s in zip(idx, st) if s > 0]
        return " + ".join(terms + (["M"] if m else []))

    m = bool(tables.is_three_body[row])
    return f"{side(tables.reactant_idx[row], tables.reactant_stoich[row], m)} -> " \
           f"{side(tables.product_idx[row], tables.product_stoich[row], m)}"


def make_rate_network(seed=0, ni=30, n_fwd=120, n_kinf=24, n_nokinf=12, n_photo=6, special=True) -> str:
    """Network text exercising every rate form of the rate build: two-body
    modified Arrhenius (``a n E``), three-body with high-pressure rates
    (Lindemann, ``a n E a_inf n_inf E_inf``), three-body without, the three
    low-temperature-cap reactions (reference `rates.py:30-33`), the special
    ``OH + CH3 + M -> CH3OH + M`` (hardcoded Troe), `# reverse stops` and a
    photo section. Reactions come from a seeded balanced network; parameters
    are seeded log-uniform / uniform draws written with 4 significant digits.
    ``special=False`` leaves out the cap and special reactions (and their
    named species), so the network has exactly ``ni`` species."""
    rng = _rng(seed, 17)
    base = make_network(seed, ni, n_fwd, n_photo=n_photo)
    t = base.tables
    rows = [r for r in range(1, t.nr + 1, 2) if not t.is_photo[r]]
    n2 = len(rows) - n_kinf - n_nokinf
    lines = ["# rate-build test network (written by jax-vulcan_b200.synthetic)", "# Two-body Reactions"]
    fid = 1

    def put(eq, cols):
        nonlocal fid
        lines.append(f"{fid:5d} [ {eq} ]  " + "  ".join(cols))
        fid += 2

    def e(x):
        return f"{x:.3E}"

    for r in rows[:n2]:
        put(_eq_of(t, r), [e(10 ** rng.uniform(-14, -9)), f"{rng.uniform(-2, 2):.3f}",
                           f"{rng.uniform(-300, 20000):.1f}"])
    lines.append("# 3-body and Disscoiation Reactions")
    for r in rows[n2:n2 + n_kinf]:
        eq = _eq_of(t, r)
        if " + M" not in eq:
            lhs, rhs = eq.split(" -> ")
            eq = f"{lhs} + M -> {rhs} + M"
        put(eq, [e(10 ** rng.uniform(-33, -26)), f"{rng.uniform(-4, 1):.3f}", f"{rng.uniform(0, 5000):.1f}",
                 e(10 ** rng.uniform(-12, -9)), f"{rng.uniform(-1, 1):.3f}", f"{rng.uniform(0, 3000):.1f}"])
    for eq in ("H + CH3 + M -> CH4 + M", "H + C2H4 + M -> C2H5 + M", "H + C2H5 + M -> C2H6 + M")[:3 * special]:
        put(eq, [e(10 ** rng.uniform(-30, -24)), f"{rng.uniform(-3, 0):.3f}", f"{rng.uniform(0, 700):.1f}",
                 e(10 ** rng.uniform(-11, -9)), f"{rng.uniform(-0.5, 1.5):.3f}", f"{rng.uniform(0, 600):.1f}"])
    lines.append("# 3-body reactions without high-pressure rates")
    for r in rows[n2 + n_kinf:]:
        eq = _eq_of(t, r)
        if " + M" not in eq:
            lhs, rhs = eq.split(" -> ")
            eq = f"{lhs} + M -> {rhs} + M"
        put(eq, [e(10 ** rng.uniform(-34, -28)), f"{rng.uniform(-3, 0):.3f}", f"{rng.uniform(0, 1000):.1f}"])
    if special:
        lines.append("# special cases")
        put("OH + CH3 + M -> CH3OH + M", [])
    lines.append("# reverse stops")
    lines.append("# photo disscoiation (no reversals)")
    for sp, br, row in base.photo_branches:
        put(_eq_of(t, row), [sp, str(br)])
    return "\n".join(lines) + "\n"


def make_nasa9(seed, ni):
    """Seeded NASA-9 coefficients [ni, 2, 10] (low-T and high-T branches,
    reference `gibbs.py:16-38` layout): magnitudes of real species' fits,
    with the enthalpy constant a8 within +-1e4 K so that g/RT stays within
    a few hundred down to 150 K."""
    rng = _rng(seed, 19)
    c = np.zeros((ni, 2, 10))
    for j in range(2):
        c[:, j, 0] = rng.uniform(-5e4, 5e4, ni)
        c[:, j, 1] = rng.uniform(-500.0, 500.0, ni)
        c[:, j, 2] = rng.uniform(2.0, 6.0, ni)
        c[:, j, 3] = rng.uniform(-5e-3, 5e-3, ni)
        c[:, j, 4] = rng.uniform(-5e-6, 5e-6, ni)
        c[:, j, 5] = rng.uniform(-3e-9, 3e-9, ni)
        c[:, j, 6] = rng.uniform(-5e-13, 5e-13, ni)
        c[:, j, 8] = rng.uniform(-1e4, 1e4, ni)
        c[:, j, 9] = rng.uniform(-10.0, 20.0, ni)
    return c


def make_balanced_rates(seed, net: SyntheticNetwork, nz, n, lo=-12.0, hi=4.0, M=None):
    """Rate constants in detailed balance with a seeded equilibrium: a network
    whose adaptive integration settles.

    The forward constants (odd rows) are order-scaled log-uniform draws
    (pseudo-first-order rates in ``[10**lo, 10**hi]`` at the densest layer,
    as `make_rates` with ``n_ref``); each reverse constant (the next row, the
    same reaction with the sides swapped) is set so that the pair's rates
    are equal at ``y* = ymix* n`` in every layer, for one seeded composition
    ``ymix*`` (log-uniform in [1e-8, 1], normalised) shared by all layers:
        k_rev = k_fwd prod_reactants y*^nu (M) / prod_products y*^nu (M).
    ``y*`` is then a steady state of the chemistry (every pair balanced, as
    Gibbs-consistent reverse rates make a thermodynamic equilibrium) and of
    eddy diffusion (uniform mixing ratios carry no flux), and a fixed point
    of the hydrostatic rebalance (its layer sums are n). Photolysis rows stay
    zero (the photo branch writes them). Returns (k [nr+1, nz], ymix* [ni]).
    """
    t = net.tables
    ni, nr = t.ni, t.nr
    n = np.asarray(n, dtype=np.float64)
    M = n if M is None else np.asarray(M, dtype=np.float64)
    rng = _rng(seed, 13)
    ymix = 10.0 ** rng.uniform(-8.0, 0.0, ni)
    ymix /= ymix.sum()
    ystar = ymix[None, :] * n[:, None]                        # [nz, ni]
    k = make_rates(seed, net, nz, lo, hi, n_ref=float(n.max()))
    ypad = np.concatenate([ystar, np.ones((nz, 1))], axis=1)   # padding index ni -> 1

    def side(r, idx, st):
        f = np.ones(nz)
        for s in range(idx.shape[1]):
            if st[r, s] > 0:
                f = f * ypad[:, idx[r, s]] ** st[r, s]
        if t.is_three_body[r]:
            f = f * M
        return f

    for r in range(1, nr, 2):
        if t.is_photo[r] or t.is_photo[r + 1]:
            continue
        assert sorted(t.reactant_idx[r + 1][t.reactant_stoich[r + 1] > 0].tolist()) == \
            sorted(t.product_idx[r][t.product_stoich[r] > 0].tolist()), "row r+1 must reverse row r"
        k[r + 1] = k[r] * side(r, t.reactant_idx, t.reactant_stoich) / side(r + 1, t.reactant_idx, t.reactant_stoich)
    return k, ymix
