"""The loop body on the GPU (``vb_loop_body`` after ``vb_ros2_step``) against
one attempt of the reference runner per fixture case (``tests/golden/body.npz``,
made by running the reference `outer_loop.py` body) and against the oracle on
batches where atmospheres take different decisions in the same launch.

Tolerances: every decision (accept / reject kind / force-accept) and counter
must be equal. The state inherits the step's error bound
``|sol - ref| <= 1e-10 |sol_ref|``: y, y_prev and ymix within 1e-10 relative;
the error norm ``delta = max(delta_arr / sol)`` within 1e-10 absolute (the
step bound divided by sol); dt, which scales as ``delta^-1/2`` unless clipped,
within ``0.5e-10 / delta`` relative; atom losses (already relative to the
initial atom totals) within 1e-10 absolute; small_y / nega_y within 1e-10
relative; t and rtol within 1e-15 relative.
"""
import numpy as np
import pytest
import torch

from conftest import BODY_FIELDS, body_kwargs, golden_body, load_pkg
from oracle import contract as oc
from oracle import ros2 as orc

pytestmark = pytest.mark.gpu

chem = load_pkg("chem")
jstep = load_pkg("jax_step")
loop = load_pkg("outer_loop")
syn = load_pkg("synthetic")

COUNTERS = ("accept_count", "retry_count", "nega_count", "loss_count", "delta_count")


def statics_of(p, kw):
    return loop.LoopStatics(**{k: p[k] for k in (
        "loss_eps", "pos_cut", "nega_cut", "mtol", "atol", "dt_var_min", "dt_var_max", "dt_min", "dt_max",
        "batch_max_retries", "use_adapt_rtol", "rtol_min", "rtol_max", "adapt_rtol_dec_period",
        "adapt_rtol_inc_period", "adapt_rtol_dec", "adapt_rtol_inc", "adapt_rtol_loss_mul",
        "adapt_rtol_inc_loss_thresh")}, zero_bot_row=kw["zero_bot_row"], hydro_partial=kw["hydro_partial"])


def state_of(inp):
    """LoopState of a batch of fixture/oracle states (list of dicts)."""
    st = lambda f: np.stack([np.asarray(s[f]) for s in inp])  # noqa: E731
    return loop.LoopState(st("y"), st("ymix"), st("dt"), st("atom_loss"), st("atom_loss_prev"),
                          y_prev=st("y_prev"), t=st("t"), rtol=st("rtol"), loss_criteria=st("loss_criteria"),
                          counters={c: st(c) for c in COUNTERS}, small_y=st("small_y"), nega_y=st("nega_y"))


def check_state(got, b, ref, what):
    for c in COUNTERS:
        assert int(got[c][b]) == int(ref[c]), (what, c, got[c][b], ref[c])

    def rel(a, r, floor=1e-300):
        return float(np.max(np.abs(np.asarray(a) - r) / np.maximum(np.abs(r), floor), initial=0.0))

    for f in ("y", "y_prev", "ymix"):
        assert rel(got[f][b], ref[f], 1e-30) <= 1e-10, (what, f, rel(got[f][b], ref[f], 1e-30))
    assert abs(float(got["delta"][b]) - ref["delta"]) <= 1e-10, (what, "delta", got["delta"][b], ref["delta"])
    dt_tol = 0.5e-10 / max(ref["delta"], 1e-300) + 1e-15
    assert rel(got["dt"][b], ref["dt"]) <= dt_tol, (what, "dt", got["dt"][b], ref["dt"])
    for f in ("atom_loss", "atom_loss_prev"):
        assert np.max(np.abs(got[f][b] - ref[f])) <= 1e-10, (what, f)
    for f in ("small_y", "nega_y"):
        assert rel(got[f][b], ref[f]) <= 1e-10, (what, f)
    for f in ("t", "rtol", "loss_criteria"):
        assert rel(got[f][b], ref[f]) <= 1e-15, (what, f, got[f][b], ref[f])


def test_loop_body_matches_reference_runner():
    net, atm, compo, atom_ini, k, params, cases = golden_body()
    dn = chem.to_device(net)
    A = jstep.atm_from_dict(atm)
    for name, c in cases.items():
        p, kw = body_kwargs(c, params)
        runner = loop.AdaptiveRunner(dn, A, statics_of(p, kw), compo, atom_ini, gas_mask=kw["gas"])
        state = state_of([c["inp"]])
        fm = fy = None
        if "fix_mask" in kw:
            fm, fy = kw["fix_mask"][None], kw["fix_y"][None]
        decisions = []
        for _ in range(len(c["hist"])):
            runner.attempt(state, k[None], fix_mask=fm, fix_y=fy)
            decisions.append(int(state.scalars_host()["last_decision"][0]))
        got = state.snapshot()
        assert [d > 0 for d in decisions] == [bool(h[0]) for h in c["hist"]], (name, decisions)
        check_state(got, 0, c["out"], name)


def test_batched_atmospheres_decide_independently():
    """vmap semantics: three atmospheres in one launch, with rtol / dt /
    retry budgets that send them down different branches on the same
    attempt, each against the oracle run on its own."""
    net, atm, compo, atom_ini, k, params, cases = golden_body()
    dn = chem.to_device(net)
    A = jstep.atm_from_dict(atm)
    base = dict(cases["accept"]["inp"])
    inp = [dict(base, rtol=0.2, dt=1e-6), dict(base, rtol=1e-3, dt=3e-5),
           dict(base, rtol=1e-30, dt=1e-6, retry_count=6)]
    p, kw = body_kwargs(cases["accept"], params)
    runner = loop.AdaptiveRunner(dn, A, statics_of(p, kw), compo, atom_ini, batch=3)
    state = state_of(inp)
    K = np.broadcast_to(k, (3,) + k.shape).copy()
    refs = [dict(s) for s in inp]
    seen = set()
    for it in range(6):
        runner.attempt(state, K)
        dec = state.scalars_host()["last_decision"]
        for b in range(3):
            refs[b] = oc.attempt(refs[b], k, atm, net, compo, atom_ini, p, **kw)
            want = 2 if refs[b]["_force"] else (1 if refs[b]["_accept"] else 0)
            assert int(dec[b]) == want, (it, b, dec, want)
            seen.add(want)
    got = state.snapshot()
    for b in range(3):
        check_state(got, b, refs[b], f"atmosphere {b}")
    assert seen == {0, 1, 2}


def test_loop_at_benchmark_shape():
    """ni=69, nz=120 (the benchmark network shape), 2 atmospheres, 3 attempts
    with rtol tight enough to reject, against the oracle."""
    case = syn.make_case(seed=31, mild=True, k_range=(-40.0, 4.0), moldiff=True)
    net, atm = case.net.tables, case.atm
    dn = chem.to_device(net)
    compo = case.net.compo
    y0 = case.y
    atom_ini = np.einsum("zi,ia->a", y0, compo) * (1 + 1e-7)
    al0 = (np.einsum("zi,ia->a", y0, compo) - atom_ini) / atom_ini
    ymix0 = y0 / y0.sum(axis=1, keepdims=True)
    s0 = dict(y=y0, y_prev=y0, ymix=ymix0, dt=1e-6, t=0.0, delta=0.0, atom_loss=al0, atom_loss_prev=al0,
              small_y=0.0, nega_y=0.0, rtol=0.05, loss_criteria=1e-3, accept_count=0, retry_count=0,
              nega_count=0, loss_count=0, delta_count=0)
    inp = [s0, dict(s0, rtol=1e-6, dt=3e-6)]
    p = dict(oc_params())
    A = {kk: (np.stack([atm[kk]] * 2) if not isinstance(atm[kk], bool) else atm[kk]) for kk in atm}
    runner = loop.AdaptiveRunner(dn, jstep.atm_from_dict(A), loop.LoopStatics(**p), compo, atom_ini, batch=2)
    state = state_of(inp)
    K = np.stack([case.k] * 2)
    refs = [dict(s) for s in inp]
    for it in range(3):
        runner.attempt(state, K)
        for b in range(2):
            refs[b] = oc.attempt(refs[b], case.k, atm, net, compo, atom_ini, dict(p, use_adapt_rtol=False))
    got = state.snapshot()
    for b in range(2):
        check_state(got, b, refs[b], f"atmosphere {b}")


def oc_params():
    return dict(loss_eps=0.1, pos_cut=0.0, nega_cut=-1.0, mtol=1e-22, atol=0.1, dt_var_min=0.5, dt_var_max=2.0,
                dt_min=1e-14, dt_max=1e4, batch_max_retries=8, rtol_min=0.02, rtol_max=1.0,
                adapt_rtol_dec_period=5, adapt_rtol_inc_period=10, adapt_rtol_dec=0.5, adapt_rtol_inc=1.5,
                adapt_rtol_loss_mul=10.0, adapt_rtol_inc_loss_thresh=1e-3)


def test_loop_body_rejects_bad_arguments():
    L = load_pkg("_lib").lib()
    p = loop.LoopStatics().params(1)
    p.n_atoms = 0
    import ctypes as C
    dummy = C.c_void_p(16)  # never dereferenced: argument checks come first
    rc = L.vb_loop_body(2, 10, 12, None, C.addressof(p), dummy, None, dummy, dummy, None, None, dummy, dummy,
                        dummy, dummy, dummy, dummy, dummy, dummy, dummy, None, None, None, None, None)
    assert rc == 1 and b"n_atoms" in L.vb_last_error()
    rc = L.vb_loop_body(2, 10, 12, None, C.addressof(p), dummy, None, dummy, dummy, dummy, None, dummy, dummy,
                        dummy, dummy, dummy, dummy, dummy, dummy, dummy, None, None, None, None, None)
    assert rc == 1 and b"fix_mask" in L.vb_last_error()


def test_loop_refresh_matches_oracle_chain():
    """The atmosphere refresh inside the loop (reference `outer_loop.py:813-840`):
    ten attempts with a refresh on every second taken attempt (pre-increment
    accept count divisible by 2) from the attempt's clipped state, g, dzi,
    Hpi and two species' escape fluxes (floored at -max_flux) written into
    the atmosphere the next step reads; against the oracle chain of the same
    attempts. Decisions equal; y and the refreshed fields within 1e-9
    relative (the step bound carried through the chain)."""
    from oracle import refresh as orf
    ar = load_pkg("atm_refresh")
    case = syn.make_case(seed=41, ni=12, n_fwd=30, nz=10, mild=True, k_range=(-40.0, 4.0), moldiff=True,
                         fluxes=True)
    tables, extra = case.net.tables, case.extra
    compo = case.net.compo
    y0 = case.y
    atom_ini = np.einsum("zi,ia->a", y0, compo) * (1 + 1e-7)
    al0 = (np.einsum("zi,ia->a", y0, compo) - atom_ini) / atom_ini
    ymix0 = y0 / y0.sum(axis=1, keepdims=True)
    esc, max_flux = np.array([0, 3]), 1e6
    st = ar.AtmRefreshStatic(pico=extra["pico"], mol_mass=case.net.ms, diff_esc_idx=esc, pref_indx=0, zco_pref=0.0,
                             gs=syn.GS, Rp=syn.RP, max_flux=max_flux)
    p = oc_params()
    runner = loop.AdaptiveRunner(chem.to_device(tables), jstep.atm_from_dict(case.atm), loop.LoopStatics(**p), compo,
                                 atom_ini, conv=loop.ConvStatics(conv_step=4, count_min=10 ** 6), refresh=st,
                                 update_frq=2, dz=extra["dz"])
    state = loop.LoopState(y0[None], ymix0[None], 1e-8, al0[None], rtol=0.2)
    atm = dict(case.atm)
    s = dict(y=y0, y_prev=y0, ymix=ymix0, dt=1e-8, t=0.0, delta=0.0, atom_loss=al0, atom_loss_prev=al0,
             small_y=0.0, nega_y=0.0, rtol=0.2, loss_criteria=1e-3, accept_count=0, retry_count=0, nega_count=0,
             loss_count=0, delta_count=0)
    refreshed = 0
    for a in range(10):
        s = oc.attempt(s, case.k, atm, tables, compo, atom_ini, dict(p, use_adapt_rtol=False))
        take = s["_accept"] or s["_force"]
        if take and (s["accept_count"] - 1) % 2 == 0:
            mu, g, Hp, dz, zco, dzi, Hpi = orf.update_mu_dz(s["_ymix_new"], atm["Tco"], extra["pico"], case.net.ms,
                                                            0, 0.0, syn.GS, syn.RP, st.kb, st.Navo)
            tf = orf.update_phi_esc(s["_sol_clip"], g, Hp, atm["top_flux"], atm["Tco"], atm["Dzz"][-1], atm["ms"],
                                    esc, st.kb, st.Navo, max_flux)
            atm.update(g=g, dzi=dzi, Hpi=Hpi, top_flux=tf)
            refreshed += 1
            last_dz = dz
        runner.attempt(state, case.k[None])
        dec = int(state.scalars_host()["last_decision"][0])
        assert dec == (2 if s["_force"] else (1 if s["_accept"] else 0)), (a, dec)
    assert refreshed >= 4
    got = state.snapshot()
    assert np.max(np.abs(got["y"][0] - s["y"]) / np.maximum(np.abs(s["y"]), 1e-30)) <= 1e-9
    f = ar.blob_fields(runner.step.blob, 10, 12)
    for name in ("g", "dzi", "Hpi", "top_flux"):
        ref = np.asarray(atm[name])
        e = np.max(np.abs(f[name][0].cpu().numpy() - ref) / np.maximum(np.abs(ref), 1e-300))
        assert e <= 1e-9, (name, e)
    assert np.max(np.abs(runner.dz[0].cpu().numpy() - last_dz) / np.abs(last_dz)) <= 1e-9


def test_loop_condensation_matches_oracle_chain():
    """Condensation inside the loop (reference `outer_loop.py:770-800`): eight
    accepted attempts, each inside the time window, so each rewrites the
    condensation rows of k (here a photolysis row, unused with photochemistry
    off) from the attempt's clipped state and relaxes species 1 toward
    saturation into species 2 with the attempt's dt, before the hydrostatic
    rebalance; against the oracle chain with the same hook. The relaxation
    moves the state by 3-25 % per attempt. Decisions equal; y, ymix and the
    atom losses within 1e-9, the condensation rows within 1e-9 relative."""
    from oracle import refresh as orf
    cd = load_pkg("conden")
    case = syn.make_case(seed=43, ni=12, n_fwd=30, nz=10, mild=True, k_range=(-40.0, 4.0), moldiff=True, n_photo=2)
    tables, compo, y0, atm = case.net.tables, case.net.compo, case.y, dict(case.atm)
    atom_ini = np.einsum("zi,ia->a", y0, compo) * (1 + 1e-7)
    al0 = (np.einsum("zi,ia->a", y0, compo) - atom_ini) / atom_ini
    ymix0 = y0 / y0.sum(axis=1, keepdims=True)
    rng = np.random.default_rng(43)
    nz = 10
    sat = y0[:, 1] * rng.uniform(0.5, 1.5, nz)
    Dg = 10 ** rng.uniform(-2, 1, nz)
    row = case.net.photo_branches[0][2]
    re_idx, sp_idx, coeff = np.array([row]), np.array([3]), np.array([1e-30])
    Dg_re = 10 ** rng.uniform(-2, 1, (1, nz))
    sat_re = y0[:, 3][None] * rng.uniform(0.5, 1.5, (1, nz))
    m = 1e-2 / (1e-8 * np.max(Dg) * np.max(y0[:, 1]))
    st = cd.CondenStatic(conden_re_idx=re_idx, conden_sp_idx=sp_idx, Dg_per_re=Dg_re[None], sat_n_per_re=sat_re[None],
                         coeff_per_re=coeff, atm_blob=None, h2o_active=True, h2o_idx=1, h2o_l_s_idx=2,
                         h2o_Dg=Dg[None], h2o_sat=sat[None], h2o_m_over_rho_r2=m, start_conden_time=0.0)
    p = oc_params()
    runner = loop.AdaptiveRunner(chem.to_device(tables), jstep.atm_from_dict(atm), loop.LoopStatics(**p), compo,
                                 atom_ini, conv=loop.ConvStatics(conv_step=4, count_min=10 ** 6), conden=st)
    state = loop.LoopState(y0[None], ymix0[None], 1e-8, al0[None], rtol=0.2)
    k = torch.as_tensor(case.k[None], device="cuda").contiguous()
    fn = lambda y, x, dt: orf.apply_relax(y, x, dt, 1, 2, Dg, sat, m, atm["M"], atm["gas_indx_mask"])  # noqa: E731
    s = dict(y=y0, y_prev=y0, ymix=ymix0, dt=1e-8, t=0.0, delta=0.0, atom_loss=al0, atom_loss_prev=al0,
             small_y=0.0, nega_y=0.0, rtol=0.2, loss_criteria=1e-3, accept_count=0, retry_count=0, nega_count=0,
             loss_count=0, delta_count=0)
    k_o = case.k.copy()
    fired = 0
    for a in range(8):
        s = oc.attempt(s, k_o, atm, tables, compo, atom_ini, dict(p, use_adapt_rtol=False),
                       conden=dict(start_time=0.0, fn=fn))
        if s["_conden_fired"]:
            k_o = orf.update_conden_rates(k_o, s["_sol_clip_raw"], re_idx, sp_idx, Dg_re, sat_re, coeff)
            fired += 1
        runner.attempt(state, k)
        dec = int(state.scalars_host()["last_decision"][0])
        assert dec == (2 if s["_force"] else (1 if s["_accept"] else 0)), (a, dec)
    assert fired == 8
    got = state.snapshot()
    for f in ("y", "ymix", "y_prev"):
        e = np.max(np.abs(got[f][0] - s[f]) / np.maximum(np.abs(s[f]), 1e-30))
        assert e <= 1e-9, (f, e)
    assert np.max(np.abs(got["atom_loss"][0] - s["atom_loss"])) <= 1e-9
    kd = k[0].cpu().numpy()
    for r in (row, row + 1):
        assert np.max(np.abs(kd[r] - k_o[r]) / np.maximum(np.abs(k_o[r]), 1e-300)) <= 1e-9, r


def test_condensation_mask_drops_species_from_the_error_norm():
    """The reference's condense_zero_mask (`outer_loop.py:244`, `:1380-1386`):
    with use_condense on, delta of the condense_sp + non_gas_sp columns is
    left out of the error norm. A delta field that is small everywhere except
    one species (above rtol there) makes the attempt a reject without the
    mask and an accept with that species masked, on the GPU as in the oracle."""
    net, atm, compo, atom_ini, k, params, cases = golden_body()
    c = cases["accept"]
    p, kw = body_kwargs(c, params)
    inp = c["inp"]
    sol, delta = orc.ros2_step(inp["y"], k, inp["dt"], atm, net)
    sol = np.abs(sol) + 1.0          # every entry counts in the norm (sol > atol, positive)
    ymix_ok = np.asarray(inp["ymix"]) >= p["mtol"]
    col = int(np.argmax(ymix_ok.all(axis=0)))
    delta = 1e-6 * np.abs(sol)
    delta[:, col] = 10.0 * inp["rtol"] * np.abs(sol[:, col])
    dn = chem.to_device(net)
    blob = jstep.pack_atm(jstep.atm_from_dict(atm))
    for masked in (False, True):
        st = statics_of(p, kw)
        if masked:
            st.cond_zero = (col,)
        state = state_of([inp])
        loop.loop_body(state, torch.as_tensor(sol[None], device="cuda"), torch.as_tensor(delta[None], device="cuda"),
                       blob, compo, atom_ini, st, gas_mask=kw["gas"])
        got = state.snapshot()
        cz = np.zeros(sol.shape[1], bool)
        if masked:
            cz[col] = True
        ref = oc.body_update(dict(inp), sol, delta, atm["M"], compo, atom_ini, dict(p), gas=kw["gas"],
                             hydro_partial=kw["hydro_partial"], zero_bot_row=kw["zero_bot_row"],
                             cond_zero=cz if masked else None)
        assert int(got["accept_count"][0]) == int(ref["accept_count"]), masked
        assert int(got["accept_count"][0]) == int(inp["accept_count"]) + (1 if masked else 0), masked
        check_state(got, 0, ref, f"cond_zero={masked}")


def test_runstate_round_trip_continues_bit_for_bit():
    """The device carry as the reference RunState runner slots (StepInputs,
    ParamInputs, AtomInputs: `state.py:106-141`) and back: after some attempts
    (at an accepted attempt, so no retry is pending), the rebuilt carry runs
    the next attempts exactly as the original does."""
    rsm = load_pkg("runstate")
    case = syn.make_case(seed=44, ni=12, n_fwd=30, nz=10, mild=True, k_range=(-40.0, 4.0), moldiff=True)
    tables, compo, y0, atm = case.net.tables, case.net.compo, case.y, case.atm
    atom_ini = np.einsum("zi,ia->a", y0, compo) * (1 + 1e-7)
    al0 = (np.einsum("zi,ia->a", y0, compo) - atom_ini) / atom_ini
    p = oc_params()
    conv = loop.ConvStatics(conv_step=4, count_min=10 ** 6)
    runner = loop.AdaptiveRunner(chem.to_device(tables), jstep.atm_from_dict(atm), loop.LoopStatics(**p), compo,
                                 atom_ini, conv=conv)
    state = loop.LoopState(y0[None], (y0 / y0.sum(axis=1, keepdims=True))[None], 1e-8, al0[None], rtol=0.2,
                           y_prev=y0[None])
    k = torch.as_tensor(case.k[None], device="cuda").contiguous()
    for _ in range(6):
        runner.attempt(state, k)
    while int(state.scalars_host()["retry_count"][0]) != 0:
        runner.attempt(state, k)
    slots = rsm.runstate_slots(state, 0, compo, ["C", "H", "O", "N"], atom_ini)
    assert set(slots["step"]) == set(rsm.STEP_FIELDS) and set(slots["params"]) == set(rsm.PARAM_FIELDS)
    assert set(slots["atoms"]) == set(rsm.ATOM_FIELDS)
    assert slots["params"]["count"] == int(state.scalars_host()["accept_count"][0])
    again = rsm.state_from_runstate([slots], rtol=0.2, conv_step=4)
    for _ in range(3):
        runner.attempt(state, k)
        runner.attempt(again, k)
    a, b = state.snapshot(), again.snapshot()
    for f in ("y", "y_prev", "ymix", "dt", "t", "atom_loss", "accept_count", "delta_count"):
        assert np.array_equal(a[f], b[f]), f
