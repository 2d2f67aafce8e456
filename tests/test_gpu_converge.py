"""The convergence chain on the GPU (``vb_loop_converge`` after
``vb_loop_body``) against 40 attempts of the reference runner
(``tests/golden/conv.npz``): ring buffer, longdy / longdydt, the stall
detector and the loop condition, and the freeze of an atmosphere once the
condition stops it.

Tolerances: counters (accept_count, retry_count, count_since_new_min) and the
stop decision must be equal. The fixture chains 40 attempts, so the step's
1e-10 relative error compounds through the carried state: t, dt, longdy,
longdydt, longdy_seen_min and the rings are held to 1e-8 relative.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden, golden_body, load_pkg

pytestmark = pytest.mark.gpu

chem = load_pkg("chem")
jstep = load_pkg("jax_step")
loop = load_pkg("outer_loop")

TOL = 1e-8


def rel(a, r, floor=1e-300):
    a, r = np.asarray(a, np.float64), np.asarray(r, np.float64)
    return float(np.max(np.abs(a - r) / np.maximum(np.abs(r), floor), initial=0.0))


def chain_setup(batch, count_min):
    net, atm, compo, atom_ini, k, params, _ = golden_body()
    g = golden("conv.npz")
    cp = {kk[len("conv_param_"):]: g[kk].item() for kk in g if kk.startswith("conv_param_")}
    p = dict(params, use_adapt_rtol=False)
    statics = loop.LoopStatics(**{kk: p[kk] for kk in (
        "loss_eps", "pos_cut", "nega_cut", "mtol", "atol", "dt_var_min", "dt_var_max", "dt_min", "dt_max",
        "batch_max_retries", "use_adapt_rtol", "rtol_min", "rtol_max", "adapt_rtol_dec_period",
        "adapt_rtol_inc_period", "adapt_rtol_dec", "adapt_rtol_inc", "adapt_rtol_loss_mul",
        "adapt_rtol_inc_loss_thresh")})
    conv = loop.ConvStatics(conv_step=4, atol=p["atol"], runtime=1e30, count_max=10 ** 6,
                            **dict(cp, count_min=count_min))
    A = jstep.atm_from_dict({kk: (np.stack([v] * batch) if not isinstance(v, bool) else v) for kk, v in atm.items()})
    runner = loop.AdaptiveRunner(chem.to_device(net), A, statics, compo, atom_ini, batch=batch, conv=conv,
                                 slope_min=float(g["conv_slope_min"]))
    rep = lambda a: np.stack([a] * batch)  # noqa: E731
    al = g["conv_in_atom_loss"]
    state = loop.LoopState(rep(g["conv_in_y"]), rep(g["conv_in_ymix"]), 1e-6, rep(al), rep(al), t=0.0, rtol=0.05,
                           loss_criteria=1e-3, small_y=1.5, nega_y=2.5)
    state.enable_convergence(4)
    return runner, state, np.stack([k] * batch), g


@pytest.mark.parametrize("count_min,first_stop", [(2, 9), (23, 24), (10 ** 6, None)])
def test_convergence_chain_matches_reference_runner(count_min, first_stop):
    """count_min 2 is the fixture's own setting (the stall detector stops the
    run at attempt 10); 23 holds the run until attempt 25, where the stall
    detector stops it again; 10**6 never stops, so all 40 attempts and the
    final rings are compared."""
    runner, state, K, g = chain_setup(1, count_min)
    n = int(g["conv_n"])
    frozen = None
    for a in range(n):
        runner.attempt(state, K)
        sc, cv = state.scalars_host()[0], state.conv_host()[0]
        if frozen is not None:
            # stopped: the body and the diagnostics leave the atmosphere alone
            assert state.y.cpu().numpy().tobytes() == frozen[0], a
            assert sc.tobytes() == frozen[1] and cv.tobytes() == frozen[2], a
            continue
        for f in ("accept_count", "retry_count"):
            assert int(sc[f]) == int(g["conv_" + f][a]), (a, f, sc[f])
        assert int(cv["count_since_new_min"]) == int(g["conv_count_since_new_min"][a]), a
        assert rel(sc["t"], g["conv_t"][a]) <= TOL, (a, "t", sc["t"], g["conv_t"][a])
        dt = state.dt.cpu().numpy()[0]
        assert rel(dt, g["conv_dt"][a]) <= TOL, (a, "dt", dt, g["conv_dt"][a])
        for f in ("longdy", "longdydt", "longdy_seen_min"):
            want = g["conv_" + f][a]
            if np.isinf(want):
                assert np.isinf(cv[f]), (a, f)
            else:
                assert rel(cv[f], want) <= TOL, (a, f, cv[f], want)
        stop = a == first_stop
        assert int(cv["done"]) == int(stop), (a, cv["done"])
        if stop:
            assert not bool(g["conv_cond"][a])
            frozen = (state.y.cpu().numpy().tobytes(), sc.tobytes(), cv.tobytes())
    if first_stop is None:
        assert rel(state.ring_y.cpu().numpy()[0], g["conv_y_ring"], 1e-30) <= TOL
        assert rel(state.ring_t.cpu().numpy()[0], g["conv_t_ring"]) <= TOL
        assert rel(state.y.cpu().numpy()[0], g["conv_y"], 1e-30) <= TOL
    assert int(state.photo_due.abs().sum()) == 0


def test_run_to_convergence_reads_back_only_per_check():
    """Two atmospheres: the stall detector stops both at attempt 10; the
    runner checks the done flags every 4 attempts, so it returns after 12
    with both frozen at the attempt-10 state."""
    runner, state, K, g = chain_setup(2, 2)
    n = runner.run_to_convergence(state, K, max_attempts=40, check_every=4)
    assert n == 12
    cv, sc = state.conv_host(), state.scalars_host()
    assert cv["done"].tolist() == [1, 1]
    assert sc["accept_count"].tolist() == [int(g["conv_accept_count"][9])] * 2
    assert rel(sc["t"], g["conv_t"][9]) <= TOL
    assert rel(cv["longdy"], g["conv_longdy"][9]) <= TOL


def test_loop_converge_rejects_bad_arguments():
    L = load_pkg("_lib").lib()
    p = loop.ConvStatics(conv_step=1).params()
    dummy = C.c_void_p(16)  # never dereferenced: argument checks come first
    rc = L.vb_loop_converge(2, 10, 12, None, C.addressof(p), dummy, dummy, None, dummy, dummy, dummy, dummy, dummy,
                            dummy, None, None)
    assert rc == 1 and b"conv_step" in L.vb_last_error()
    p = loop.ConvStatics(conv_step=4).params()
    rc = L.vb_loop_converge(2, 10, 12, None, C.addressof(p), dummy, dummy, None, dummy, dummy, dummy, None, dummy,
                            dummy, None, None)
    assert rc == 1 and b"null" in L.vb_last_error()
    torch.cuda.synchronize()


def test_photo_branch_inside_the_loop_matches_oracle_chain():
    """Ten attempts with photochemistry on (30 species, 10 photolysis
    branches, nz=12, 1700 bins): the photo cadence (first attempt due, then
    ``accept_count % update_photo_frq == 0`` with no retry pending), the
    switch from the initial (3) to the final (2) frequency, the photolysis
    rows of k, the actinic-flux change and the state, against the oracle
    chain of the same attempts (photo kernels, body, convergence). The chain
    accepts, rejects and skips due photo updates behind retries. The
    actinic-flux change (here ~1e-6, a ratio of differences of fluxes good to
    ~1e-12) is held to 1e-10 absolute plus 1e-8 relative."""
    from oracle import contract as oc
    from oracle import photo as op
    photo = load_pkg("photo")
    syn = load_pkg("synthetic")
    net = syn.make_network(7, 30, 185, n_photo=10)
    case = syn.make_case(seed=7, net=net, nz=12, mild=True, k_range=(-20.0, -2.0))
    bins, din12 = syn.make_bins(bin_max=402.0)
    ph = dict(syn.make_photo(7, net, case.atm["Tco"], bins, din12), f_diurnal=1e-3)
    tables, atm, dz = net.tables, case.atm, case.extra["dz"]
    nz, nbin = case.y.shape[0], bins.shape[0]
    compo = net.compo
    y0 = case.y
    atom_ini = np.einsum("zi,ia->a", y0, compo) * (1 + 1e-7)
    al0 = (np.einsum("zi,ia->a", y0, compo) - atom_ini) / atom_ini
    ymix0 = y0 / y0.sum(axis=1, keepdims=True)
    body = dict(loss_eps=0.1, pos_cut=0.0, nega_cut=-1.0, mtol=1e-22, atol=0.1, dt_var_min=0.5, dt_var_max=2.0,
                dt_min=1e-14, dt_max=1e4, batch_max_retries=8, rtol_min=0.02, rtol_max=1.0,
                adapt_rtol_dec_period=5, adapt_rtol_inc_period=10, adapt_rtol_dec=0.5, adapt_rtol_inc=1.5,
                adapt_rtol_loss_mul=10.0, adapt_rtol_inc_loss_thresh=1e-3)
    cs = loop.ConvStatics(conv_step=4, count_min=10 ** 6, use_photo=True, ini_update_photo_frq=3,
                          final_update_photo_frq=2, photo_switch_longdy=1e300, photo_switch_longdydt=1e300)
    p = dict(body, use_adapt_rtol=False, **{f: getattr(cs, f) for f in (
        "conv_step", "count_min", "count_max", "conv_stall_window", "st_factor", "mtol_conv", "yconv_cri",
        "yconv_min", "slope_cri", "flux_cri", "trun_min", "runtime", "use_photo", "final_update_photo_frq",
        "photo_switch_longdy", "photo_switch_longdydt")})
    dev = photo.PhotoDevice(ph, nz)
    runner = loop.AdaptiveRunner(chem.to_device(tables), jstep.atm_from_dict(atm), loop.LoopStatics(**body), compo,
                                 atom_ini, conv=cs, slope_min=1e-8, photo=dev, dz=dz, flux_atol=1.0)
    state = loop.LoopState(y0[None], ymix0[None], 1e-6, al0[None], rtol=0.05)
    runner.start(state)
    k = torch.as_tensor(case.k[None], device="cuda").contiguous()

    s = dict(y=y0, y_prev=y0, ymix=ymix0, dt=1e-6, t=0.0, delta=0.0, accept_count=0, retry_count=0,
             atom_loss=al0, atom_loss_prev=al0, nega_count=0, loss_count=0, delta_count=0, small_y=0.0, nega_y=0.0,
             rtol=0.05, loss_criteria=1e-3, longdy=1.0, longdydt=1.0, longdy_seen_min=np.inf,
             count_since_new_min=0, update_photo_frq=3, is_final_photo_frq=False, aflux_change=0.0)
    kr, aflux, du = case.k.copy(), np.zeros((nz, nbin)), np.zeros((nz + 1, nbin))
    ring_y, ring_t = np.zeros((4, nz, tables.ni)), np.zeros(4)
    due, n_photo = True, 0
    for a in range(10):
        assert int(state.photo_due.cpu()[0]) == int(due), a
        if due:
            n_photo += 1
            kr, anew, du = op.photo_update(s["y"], s["ymix"], dz, kr, ph, du)
            s["aflux_change"] = op.aflux_change(anew, aflux, 1.0)
            aflux = anew
        s = oc.attempt(s, kr, atm, tables, compo, atom_ini, p)
        s.update(oc.conv_update(s, ring_y, ring_t, atm["M"], p, do_accept=s["_accept"] or s["_force"]))
        s.update(oc.photo_switch(s, p))
        done = not oc.loop_continues(s, p, 1e-8, s["aflux_change"])
        due = (not done) and oc.photo_due(s, p)
        runner.attempt(state, k)
        sc, cv = state.scalars_host()[0], state.conv_host()[0]
        assert rel(k[0].cpu().numpy(), kr, 1e-300) <= TOL, a
        assert abs(cv["aflux_change"] - s["aflux_change"]) <= 1e-10 + TOL * s["aflux_change"], \
            (a, cv["aflux_change"], s["aflux_change"])
        for f in ("accept_count", "retry_count", "count_since_new_min", "update_photo_frq"):
            assert int(sc[f] if f in sc.dtype.names else cv[f]) == int(s[f]), (a, f)
        assert int(cv["is_final_photo_frq"]) == int(s["is_final_photo_frq"]) and int(cv["done"]) == int(done)
        assert rel(state.y.cpu().numpy()[0], s["y"], 1e-30) <= TOL, a
        assert rel(sc["t"], s["t"]) <= TOL and rel(cv["longdy"], s["longdy"]) <= TOL, a
    assert rel(runner.photo_carry.aflux[0].cpu().numpy(), aflux, 1e-300) <= TOL
    assert n_photo >= 3


def test_loop_reaches_the_known_steady_state():
    """The open chain 0 -> A -> B -> 0 of the reference's steady-state tests
    (k1=1, k3=0.5, k5=0.3, four layers, eddy and molecular diffusion): the
    device loop (step, body, convergence) runs from a uniform 1:1 state until
    its own loop condition stops it, and the state it stops at is the
    reference's Newton steady state (``tests/golden/adjoint.npz``; close to
    the well-mixed [A] = k1/k3 = 2, [B] = k1/k5 = 10/3, with boundary layers
    off by ~0.4 %). The body rescales every accepted state to n_0 * ymix, so
    the layer densities n_0 = M are set to the steady state's layer totals:
    M enters only three-body chemistry (none here), so this leaves the steady
    state unchanged and makes it a fixed point of the loop. Stopping rule:
    longdy < 1e-7 with longdydt < 1e-9 over the lookback window, so the
    stopped state is within 1e-5 of the steady state."""
    g = golden("adjoint.npz")
    NT = load_pkg("network").NetworkTables
    net = NT(species=("A", "B"), ni=2, nr=6, reactant_idx=g["chain_r_idx"], product_idx=g["chain_p_idx"],
             reactant_stoich=g["chain_r_st"], product_stoich=g["chain_p_st"], is_three_body=g["chain_three"],
             is_photo=np.zeros(7, bool))
    nz, ni = 4, 2
    n0 = g["chain_y"].sum(axis=1)
    atm = dict(Kzz=np.full(nz - 1, 1e-2), Dzz=np.full((nz - 1, ni), 1e-3), dzi=np.full(nz - 1, 1.0),
               vz=np.zeros(nz - 1), Hpi=np.full(nz - 1, 1.0), Ti=np.full(nz - 1, 1500.0), Tco=np.full(nz, 1500.0),
               g=np.full(nz, 1.0), ms=np.full(ni, 1.0), alpha=np.zeros(ni), M=n0.copy(),
               vm=np.zeros((nz, ni)), vs=np.zeros((nz - 1, ni)), top_flux=np.zeros(ni), bot_flux=np.zeros(ni),
               bot_vdep=np.zeros(ni), gas_indx_mask=np.ones(ni, dtype=bool), use_vm_mol=False,
               use_settling=False, use_topflux=False, use_botflux=False)
    k = np.zeros((1, 7, nz))
    k[0, 1], k[0, 3], k[0, 5] = 1.0, 0.5, 0.3
    y0 = np.repeat((n0 / 2.0)[None, :, None], ni, axis=2)
    compo = np.ones((ni, 1))
    atom_ini = y0[0].sum(axis=0) @ compo
    statics = loop.LoopStatics(loss_eps=1e30, dt_max=1e3)      # open chain: atoms are not conserved
    conv = loop.ConvStatics(conv_step=50, count_min=100, yconv_cri=1e-7, slope_cri=1e-9, yconv_min=1e-7,
                            trun_min=1.0, runtime=1e12, count_max=20000)
    runner = loop.AdaptiveRunner(chem.to_device(net), jstep.atm_from_dict(atm), statics, compo, atom_ini,
                                 conv=conv, slope_min=1e-10)
    state = loop.LoopState(y0, np.full_like(y0, 0.5), 1e-3, np.zeros((1, 1)), rtol=0.05)
    n = runner.run_to_convergence(state, k, max_attempts=20000, check_every=100)
    sc, cv = state.scalars_host()[0], state.conv_host()[0]
    assert cv["done"] == 1 and sc["accept_count"] < 20000 and sc["t"] < 1e12, (n, sc, cv)
    assert cv["longdy"] < 1e-7 and cv["longdydt"] < 1e-9      # stopped by convergence, not by a cap
    y = state.y.cpu().numpy()[0]
    assert rel(y, g["chain_y"]) <= 1e-5, (y, g["chain_y"])
    assert rel(y[:, 0], np.full(nz, 2.0)) <= 1e-2 and rel(y[:, 1], np.full(nz, 10.0 / 3.0)) <= 1e-2


def test_checkpoint_resume_is_bit_exact(tmp_path):
    """Checkpoint and resume of the device loop: a run with photochemistry
    and convergence stops after 6 attempts, is saved (carry, records, rings,
    photo-due flags, k, the packed atmosphere, the photo carry), and a fresh
    runner that loads the checkpoint continues 6 attempts to the same bits
    as the original run continuing without a stop."""
    photo = load_pkg("photo")
    syn = load_pkg("synthetic")
    net = syn.make_network(7, 30, 185, n_photo=10)
    case = syn.make_case(seed=7, net=net, nz=12, mild=True, k_range=(-20.0, -2.0))
    bins, din12 = syn.make_bins(bin_max=402.0)
    ph = dict(syn.make_photo(7, net, case.atm["Tco"], bins, din12), f_diurnal=1e-3)
    compo, y0 = net.compo, case.y
    atom_ini = np.einsum("zi,ia->a", y0, compo) * (1 + 1e-7)
    al0 = (np.einsum("zi,ia->a", y0, compo) - atom_ini) / atom_ini
    ymix0 = y0 / y0.sum(axis=1, keepdims=True)
    body = dict(loss_eps=0.1, pos_cut=0.0, nega_cut=-1.0, mtol=1e-22, atol=0.1, dt_var_min=0.5, dt_var_max=2.0,
                dt_min=1e-14, dt_max=1e4, batch_max_retries=8, rtol_min=0.02, rtol_max=1.0,
                adapt_rtol_dec_period=5, adapt_rtol_inc_period=10, adapt_rtol_dec=0.5, adapt_rtol_inc=1.5,
                adapt_rtol_loss_mul=10.0, adapt_rtol_inc_loss_thresh=1e-3)
    cs = loop.ConvStatics(conv_step=4, count_min=10 ** 6, use_photo=True, ini_update_photo_frq=3,
                          final_update_photo_frq=2, photo_switch_longdy=1e300, photo_switch_longdydt=1e300)

    def make_runner():
        return loop.AdaptiveRunner(chem.to_device(net.tables), jstep.atm_from_dict(case.atm),
                                   loop.LoopStatics(**body), compo, atom_ini, conv=cs, slope_min=1e-8,
                                   photo=photo.PhotoDevice(ph, 12), dz=case.extra["dz"], flux_atol=1.0)

    carry_fields = ("tau", "aflux", "sflux", "dflux_d", "dflux_u", "J_br", "J_br_T")
    ra = make_runner()
    sa = loop.LoopState(y0[None], ymix0[None], 1e-6, al0[None], rtol=0.05)
    ra.start(sa)
    ka = torch.as_tensor(case.k[None], device="cuda").contiguous()
    for _ in range(6):
        ra.attempt(sa, ka)
    path = tmp_path / "loop.npz"
    sa.save(path, k=ka, blob=ra.step.blob, **{f: getattr(ra.photo_carry, f) for f in carry_fields})
    for _ in range(6):
        ra.attempt(sa, ka)
    torch.cuda.synchronize()

    rb = make_runner()
    sb, extra = loop.LoopState.load(path)
    kb = extra["k"].contiguous()
    rb.step.blob.copy_(extra["blob"])
    for f in carry_fields:
        getattr(rb.photo_carry, f).copy_(extra[f])
    for _ in range(6):
        rb.attempt(sb, kb)
    torch.cuda.synchronize()
    for f in ("y", "y_prev", "ymix", "dt", "atom_loss", "atom_loss_prev", "scalars", "conv", "ring_y", "ring_t",
              "photo_due"):
        assert torch.equal(getattr(sa, f), getattr(sb, f)), f
    assert torch.equal(ka, kb)
    for f in carry_fields:
        assert torch.equal(getattr(ra.photo_carry, f), getattr(rb.photo_carry, f)), f
    assert int(sa.scalars_host()["accept_count"][0]) >= 8


def test_relaxing_network_runs_to_the_reference_stop_like_the_oracle():
    """A network that settles (30 species, 185+185 reactions, nz=40): the
    reverse constants are in detailed balance with a seeded equilibrium
    composition (``synthetic.make_balanced_rates``), the start is that
    composition with each mixing ratio scaled by up to 2x. The device loop
    (step, body, convergence) and the oracle chain (the reference body and
    cond_fn restated) both run with the reference's stopping rule
    (vulcan_cfg: yconv_cri 0.01, yconv_min 0.1, slope_cri 1e-4, trun_min 1e2)
    with count_min lowered from 120 to 50, until their own loop condition
    stops them. They must stop at the same attempt with the same counters,
    the same final mixing ratios (1e-6 relative where ymix > 1e-20) and atom
    losses (1e-6 relative: the two stop at atom losses of ~0.034 that agree
    to 3.6e-7).

    Why count_min 50: this network is settled after about 71 accepted steps
    (longdy 1.6e-3, dt 1.4e6 s). Held to count_min 120, both loops keep
    stepping with dt growing past 1e10 s, where I/(gamma dt) - J is singular
    to working precision along the atom-conserving directions; round-off is
    amplified by ~gamma dt |J| per step, the oracle chain itself wanders
    (atom loss ~0.2, longdy 0.1-1) and stops at whatever attempt longdy
    dips under yconv_min. Two correct FP64 implementations with different
    summation orders then stop at different attempts, so that regime has no
    attempt-exact answer to compare."""
    from oracle import contract as oc
    syn = load_pkg("synthetic")
    net = syn.make_network(60, 30, 185)
    nz = 40
    atm, ex = syn.make_atmosphere(60, net, nz=nz)
    k, ymix_eq = syn.make_balanced_rates(60, net, nz, ex["n"], M=atm["M"])
    rng = np.random.default_rng(1)
    ymix0 = ymix_eq * 10.0 ** rng.uniform(-0.3, 0.3, ymix_eq.shape)
    ymix0 = ymix0 / ymix0.sum()
    y0 = ymix0[None] * ex["n"][:, None]
    compo = net.compo
    atom_ini = np.einsum("zi,ia->a", y0, compo)
    al0 = np.zeros(compo.shape[1])
    body = dict(loss_eps=0.1, pos_cut=0.0, nega_cut=-1.0, mtol=1e-22, atol=0.1, dt_var_min=0.5, dt_var_max=2.0,
                dt_min=1e-14, dt_max=1e17, batch_max_retries=8, rtol_min=0.02, rtol_max=1.0,
                adapt_rtol_dec_period=5, adapt_rtol_inc_period=10, adapt_rtol_dec=0.5, adapt_rtol_inc=1.5,
                adapt_rtol_loss_mul=10.0, adapt_rtol_inc_loss_thresh=1e-3)
    cs = loop.ConvStatics(count_min=50)
    p = dict(body, use_adapt_rtol=False, **{f: getattr(cs, f) for f in (
        "conv_step", "count_min", "count_max", "conv_stall_window", "st_factor", "mtol_conv", "yconv_cri",
        "yconv_min", "slope_cri", "flux_cri", "trun_min", "runtime", "use_photo", "final_update_photo_frq",
        "photo_switch_longdy", "photo_switch_longdydt")})
    sm = float(loop.slope_min_of(atm["Kzz"], ex["Hp"])[0])
    # oracle chain to its own stop
    s = dict(y=y0, y_prev=y0, ymix=np.broadcast_to(ymix0, y0.shape).copy(), dt=1e-10, t=0.0, delta=0.0,
             accept_count=0, retry_count=0, atom_loss=al0, atom_loss_prev=al0, nega_count=0, loss_count=0,
             delta_count=0, small_y=0.0, nega_y=0.0, rtol=0.2, loss_criteria=1e-3, longdy=1.0, longdydt=1.0,
             longdy_seen_min=np.inf, count_since_new_min=0)
    ring_y, ring_t = np.zeros((cs.conv_step, nz, net.tables.ni)), np.zeros(cs.conv_step)
    n_oracle = 0
    while n_oracle < 2000:
        s = oc.attempt(s, k, atm, net.tables, compo, atom_ini, p)
        s.update(oc.conv_update(s, ring_y, ring_t, atm["M"], p, do_accept=s["_accept"] or s["_force"]))
        n_oracle += 1
        if not oc.loop_continues(s, p, sm):
            break
    assert n_oracle < 2000 and s["longdy"] < cs.yconv_cri, (n_oracle, s["longdy"])
    # the device loop to its own stop
    runner = loop.AdaptiveRunner(chem.to_device(net.tables), jstep.atm_from_dict(atm), loop.LoopStatics(**body), compo,
                                 atom_ini, conv=cs, slope_min=sm)
    state = loop.LoopState(y0[None], np.broadcast_to(ymix0, y0.shape)[None], 1e-10, al0[None], rtol=0.2)
    n_dev = runner.run_to_convergence(state, k[None], max_attempts=2000, check_every=1)
    sc, cv = state.scalars_host()[0], state.conv_host()[0]
    assert cv["done"] == 1 and n_dev == n_oracle, (n_dev, n_oracle)
    for f in ("accept_count", "retry_count", "delta_count", "loss_count"):
        assert int(sc[f]) == int(s[f]), f
    ym = state.ymix.cpu().numpy()[0]
    mask = s["ymix"] > 1e-20
    assert np.max(np.abs(ym - s["ymix"])[mask] / s["ymix"][mask]) <= 1e-6
    al = state.atom_loss.cpu().numpy()[0]
    assert np.max(np.abs(al - s["atom_loss"]) / np.maximum(np.abs(s["atom_loss"]), 1e-6)) <= 1e-6
    assert rel(sc["t"], s["t"]) <= 1e-6
