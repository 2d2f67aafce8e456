"""Generate the golden fixtures by running the REFERENCE's own code.

Run in the build container (the reference sources are not on the GPU box):

    python tests/golden/make_golden.py --reference <reference checkout>

(or with the checkout's path in $VULCAN_REFERENCE).

JAX is not installed, so the unmodified reference modules (`network.py`,
`chem.py`, `solver.py`, `jax_step.py`, `photo.py`, `integrate.py`,
`steady_state_grad.py`, `rates.py`, `gibbs.py`, `atm_refresh.py`,
`conden.py`, and the caller-contract functions of `outer_loop.py`)
are imported with ``_jax_numpy_shim`` standing in for ``jax``. A stub
``vulcan_cfg`` with no species lists is installed first so the reference
parser does not append config-named species (reference `network.py:157-194`).

Inputs are the package's seeded synthetic cases at small sizes; every input
array is stored next to the reference output so the fixtures do not depend
on the generator reproducing bit-identical floats elsewhere.
"""
from __future__ import annotations

import __future__
import argparse
import ast
import importlib
import os
import sys
import tempfile
import types
from typing import NamedTuple, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, REPO)

ATM_KEYS = ["Kzz", "Dzz", "dzi", "vz", "Hpi", "Ti", "Tco", "g", "ms", "alpha", "M", "vm", "vs",
            "top_flux", "bot_flux", "bot_vdep", "gas_indx_mask"]
FLAG_KEYS = ["use_vm_mol", "use_settling", "use_topflux", "use_botflux"]
TABLE_KEYS = ["reactant_idx", "product_idx", "reactant_stoich", "product_stoich", "is_three_body"]


def load_reference(ref):
    import _jax_numpy_shim as shim
    shim.install()
    sys.modules["vulcan_cfg"] = types.ModuleType("vulcan_cfg")
    sys.path.insert(0, ref)
    mods = {m: importlib.import_module(m) for m in
            ["network", "chem", "solver", "jax_step", "photo", "integrate", "steady_state_grad"]}
    # caller-contract functions of outer_loop.py, compiled from the reference source
    src = open(os.path.join(ref, "outer_loop.py")).read()
    tree = ast.parse(src)
    want = {"_compute_atom_loss", "_step_size", "_make_clip_fn", "_make_aggregate_delta_fn"}
    body = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in want]
    ns = {"jnp": shim.jnp, "jax": shim.jax, "np": np}
    exec(compile(ast.Module(body=body, type_ignores=[]), "outer_loop.py", "exec"), ns)
    mods["contract"] = types.SimpleNamespace(**{k: ns[k] for k in want})
    return mods, shim


def ref_atm(mods, atm):
    kw = {k: np.asarray(atm[k]) for k in ATM_KEYS}
    kw.update({k: bool(atm[k]) for k in FLAG_KEYS})
    return mods["jax_step"].AtmStatic(**kw)


def step_fixture(mods, name, case, fix_mask=None, n_steps=0):
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(case.net.text)
        path = f.name
    rn = mods["network"].parse_network(path)
    os.unlink(path)
    net = mods["chem"].to_jax(rn)
    atm = ref_atm(mods, case.atm)
    sol, delta = mods["jax_step"].jax_ros2_step(case.y, case.k, case.dt, atm, net, fix_mask=fix_mask)
    rhs = mods["chem"].chem_rhs(case.y, case.atm["M"], case.k, net)
    jac = mods["chem"].chem_jac_analytical(case.y, case.atm["M"], case.k, net)
    out = dict(net_text=np.array(case.net.text), y=case.y, k=case.k, dt=np.array(case.dt),
               sol=np.asarray(sol), delta=np.asarray(delta), rhs=np.asarray(rhs), jac=np.asarray(jac),
               ni=np.array(rn.ni), nr=np.array(rn.nr), compo=case.net.compo)
    for k in TABLE_KEYS:
        out["tab_" + k] = np.asarray(getattr(rn, k))
    for k in ATM_KEYS + FLAG_KEYS:
        out["atm_" + k] = np.asarray(case.atm[k])
    if fix_mask is not None:
        out["fix_mask"] = fix_mask
    if n_steps:
        yN, deltas = mods["integrate"].jax_integrate_fixed_dt(case.y, case.k, case.dt, n_steps, atm, net)
        out["int_y"] = np.asarray(yN)
        out["int_deltas"] = np.asarray(deltas)
        out["int_n"] = np.array(n_steps)
    np.savez_compressed(os.path.join(HERE, f"step_{name}.npz"), **out)
    print(f"step_{name}: ni={rn.ni} nr={rn.nr} nz={case.y.shape[0]}")


def thomas_fixture(mods):
    """The seeded systems of reference tests/test_block_thomas.py:22-79 and
    tests/test_block_thomas_diag.py:40-120, solved by the reference solver."""
    solver = mods["solver"]
    out = {}
    rng = np.random.default_rng(42)
    nz, ni = 8, 5
    d = rng.standard_normal((nz, ni, ni)) + 10.0 * np.eye(ni)
    sp = rng.standard_normal((nz - 1, ni, ni))
    sb = rng.standard_normal((nz - 1, ni, ni))
    r = rng.standard_normal((nz, ni))
    out.update(dense_small_diag=d, dense_small_sup=sp, dense_small_sub=sb, dense_small_rhs=r,
               dense_small_x=np.asarray(solver.block_thomas(d, sp, sb, r)))
    rng = np.random.default_rng(7)
    d = rng.standard_normal((nz, ni, ni)) + 10.0 * np.eye(ni)
    su = rng.standard_normal((nz - 1, ni))
    sb = rng.standard_normal((nz - 1, ni))
    r = rng.standard_normal((nz, ni))
    out.update(diag_small_diag=d, diag_small_sup=su, diag_small_sub=sb, diag_small_rhs=r,
               diag_small_x=np.asarray(solver.block_thomas_diag_offdiag(d, su, sb, r)))
    nz2, ni2 = 120, 93
    d2 = rng.standard_normal((nz2, ni2, ni2)) + 1e10 * np.eye(ni2)
    su2 = rng.standard_normal((nz2 - 1, ni2)) * 1e-3
    sb2 = rng.standard_normal((nz2 - 1, ni2)) * 1e-3
    r2 = rng.standard_normal((nz2, ni2))
    out.update(diag_big_x=np.asarray(solver.block_thomas_diag_offdiag(d2, su2, sb2, r2)),
               diag_big_checksum=np.array([d2.sum(), su2.sum(), sb2.sum(), r2.sum()]))
    np.savez_compressed(os.path.join(HERE, "thomas.npz"), **out)
    print("thomas: ok")


def contract_fixture(mods):
    c = mods["contract"]
    rng = np.random.default_rng(17)
    nz, ni, na = 10, 12, 4
    sol = rng.normal(0, 1, (nz, ni)) * 10.0 ** rng.uniform(-30, 5, (nz, ni))
    delta = np.abs(rng.normal(0, 1, (nz, ni))) * np.abs(sol) * 10.0 ** rng.uniform(-4, 0, (nz, ni))
    ymix_old = 10.0 ** rng.uniform(-26, 0, (nz, ni))
    compo = rng.integers(0, 4, (ni, na)).astype(np.float64)
    atom_ini = np.abs(rng.normal(10, 1, na)) * 1e20
    gas = rng.random(ni) > 0.2
    clip_g = c._make_clip_fn(True, gas, 1e-22, 0.0, -1.0)
    clip_a = c._make_clip_fn(False, gas, 1e-22, 0.0, -1.0)
    yg, mg, sg, ng = clip_g(sol, ymix_old)
    ya, ma, sa, na_ = clip_a(sol, ymix_old)
    cz = rng.random((nz, ni)) < 0.1
    agg = c._make_aggregate_delta_fn(1e-22, 1e-1, False, np.zeros((nz, ni), bool))
    agg_b = c._make_aggregate_delta_fn(1e-22, 1e-1, True, cz)
    dts = 10.0 ** rng.uniform(-12, -2, 32)
    deltas = np.concatenate([[0.0], 10.0 ** rng.uniform(-6, 2, 31)])
    h = np.array([c._step_size(dt, dl, 0.2, 0.5, 2.0, 1e-14, 1e-2) for dt, dl in zip(dts, deltas)])
    al = np.asarray(c._compute_atom_loss(np.abs(sol), compo, atom_ini))
    np.savez_compressed(os.path.join(HERE, "contract.npz"), sol=sol, delta=delta, ymix_old=ymix_old,
                        compo=compo, atom_ini=atom_ini, gas=gas, cz=cz,
                        clip_gas_y=np.asarray(yg), clip_gas_mix=np.asarray(mg),
                        clip_gas_small=np.asarray(sg), clip_gas_nega=np.asarray(ng),
                        clip_all_y=np.asarray(ya), clip_all_mix=np.asarray(ma),
                        clip_all_small=np.asarray(sa), clip_all_nega=np.asarray(na_),
                        agg=np.asarray(agg(np.asarray(yg), delta, ymix_old)),
                        agg_bot=np.asarray(agg_b(np.asarray(yg), delta, ymix_old)),
                        dts=dts, deltas=deltas, dt_next=h, atom_loss=al)
    print("contract: ok")


BODY_FIELDS = ["y", "y_prev", "ymix", "dt", "t", "delta", "accept_count", "retry_count", "atom_loss",
               "atom_loss_prev", "nega_count", "loss_count", "delta_count", "small_y", "nega_y", "rtol",
               "loss_criteria"]


def load_runner(ref, mods, shim):
    """`_make_runner` of outer_loop.py with its state/statics types, compiled
    from the reference source. `jax.jit` is the identity and
    `jax.lax.while_loop` runs the body exactly once, so one runner call is one
    accept / reject / force-accept attempt of the reference loop
    (`outer_loop.py:715-1100`)."""
    src = open(os.path.join(ref, "outer_loop.py")).read()
    tree = ast.parse(src)
    want = {"JaxIntegState", "_Statics", "_compute_atom_loss", "_step_size", "_make_clip_fn",
            "_make_aggregate_delta_fn", "_make_runner"}
    body = [n for n in tree.body if isinstance(n, (ast.FunctionDef, ast.ClassDef)) and n.name in want]
    lax_once = types.SimpleNamespace(while_loop=lambda cond, fn, init: fn(init))
    ns = {"jnp": shim.jnp, "jax": types.SimpleNamespace(jit=lambda f: f, lax=lax_once), "np": np,
          "NamedTuple": NamedTuple, "Optional": Optional,
          "jax_ros2_step": mods["jax_step"].jax_ros2_step, "AtmStatic": mods["jax_step"].AtmStatic}
    code = compile(ast.Module(body=body, type_ignores=[]), "outer_loop.py", "exec",
                   flags=__future__.annotations.compiler_flag, dont_inherit=True)
    exec(code, ns)
    return ns


BODY_PARAMS = dict(loss_eps=0.1, pos_cut=0.0, nega_cut=-1.0, mtol=1e-22, atol=0.1, dt_var_min=0.5,
                   dt_var_max=2.0, dt_min=1e-14, dt_max=1e4, batch_max_retries=8, use_adapt_rtol=False,
                   rtol_min=0.02, rtol_max=1.0, adapt_rtol_dec_period=5, adapt_rtol_inc_period=10,
                   adapt_rtol_dec=0.5, adapt_rtol_inc=1.5, adapt_rtol_loss_mul=10.0,
                   adapt_rtol_inc_loss_thresh=1e-3, use_fix_species=False, post_conden_rtol=0.2)


def body_fixture(mods, syn, ref, shim):
    """One attempt of the reference adaptive loop per case, from a state we
    choose, covering accept, the three reject kinds, both force-accept
    triggers, the gas-only hydrostatic rebalance, fixed species, the
    bottom-row mask, adaptive rtol, plus a chain of attempts."""
    ns = load_runner(ref, mods, shim)
    JS, ST = ns["JaxIntegState"], ns["_Statics"]
    J = lambda a: np.asarray(a).view(shim.JArr)  # noqa: E731
    case = syn.make_case(seed=6, ni=12, n_fwd=30, nz=10, moldiff=True, fluxes=True, mild=True,
                         k_range=(-40.0, 4.0))
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(case.net.text)
        path = f.name
    rn = mods["network"].parse_network(path)
    os.unlink(path)
    net = mods["chem"].to_jax(rn)
    atm = ref_atm(mods, case.atm)
    nz, ni = case.y.shape
    compo = case.net.compo
    y0 = case.y.copy()
    atom_ini = np.einsum("zi,ia->a", y0, compo) * 1.0000001
    conv_step = 4

    def statics(p):
        f = {k: None for k in ST._fields}
        f.update(compo_arr=J(compo), atom_ini_arr=J(atom_ini), initial_rtol=0.2, conv_step=conv_step,
                 count_min=1, count_max=10 ** 6, conv_stall_window=10 ** 6, runtime=1e30, trun_min=0.0,
                 st_factor=0.5, yconv_cri=0.01, yconv_min=0.1, slope_cri=1e-4, flux_cri=0.1,
                 mtol_conv=1e-20, conver_ignore_mask=J(np.zeros(ni, bool)),
                 condense_zero_conv_mask=J(np.zeros((nz, ni), bool)), n_0=J(case.atm["M"]),
                 Kzz=J(case.atm["Kzz"]), use_photo=False, use_atm_refresh=False, use_conden=False,
                 ini_update_photo_frq=1, final_update_photo_frq=1, update_frq=1,
                 initial_loss_criteria=1e-3, photo_switch_longdy_thresh=0.0,
                 photo_switch_longdydt_thresh=0.0, hycean_pin_time=1e30, use_ion=False, e_idx=0,
                 charge_arr=J(np.zeros(ni)), use_fix_all_bot=False, bottom_n=J(np.zeros(ni)),
                 use_fix_sp_bot=False, fix_sp_bot_idx=J(np.zeros(0, np.int32)),
                 fix_sp_bot_mix=J(np.zeros(0)), use_fix_H2He=False, h2_idx=-1, he_idx=-1,
                 fix_species_from_coldtrap_lev=False, fix_species_idx=J(np.zeros(0, np.int32)),
                 fix_species_sat_mix=J(np.zeros((0, nz))), fix_species_wholecol=J(np.zeros(0, bool)),
                 save_evolution=False, save_evo_frq=1, save_evo_n_max=1)
        f.update(p)
        return ST(**f)

    def mix(y, gas=None):
        g = np.ones(ni, bool) if gas is None else gas
        return y / np.sum(np.where(g[None, :], y, 0.0), axis=1, keepdims=True)

    def state(y, ymix, dt, rtol, **over):
        al = (np.einsum("zi,ia->a", y, compo) - atom_ini) / atom_ini
        f = {k: None for k in JS._fields}
        z2 = J(np.zeros((1, 1)))
        f.update(y=J(y), y_prev=J(y), ymix=J(ymix), dt=np.float64(dt), t=np.float64(1e3),
                 delta=np.float64(0.0), accept_count=np.int32(7), retry_count=np.int32(0), atom_loss=J(al),
                 atom_loss_prev=J(al), nega_count=np.int32(1), loss_count=np.int32(2),
                 delta_count=np.int32(3), small_y=np.float64(1.5), nega_y=np.float64(2.5), k_arr=J(case.k),
                 tau=z2, aflux=z2, sflux=z2, dflux_d=z2, dflux_u=z2, prev_aflux=z2,
                 aflux_change=np.float64(0.0), J_br=z2, J_br_T=z2, Jion_br=z2, g=J(case.atm["g"]),
                 mu=J(np.ones(nz)), Hp=J(np.ones(nz)), dz=J(np.ones(nz)), zco=J(np.zeros(nz + 1)),
                 dzi=J(case.atm["dzi"]), Hpi=J(case.atm["Hpi"]), top_flux=J(case.atm["top_flux"]),
                 vs=J(case.atm["vs"]), y_time_ring=J(np.zeros((conv_step, nz, ni))),
                 t_time_ring=J(np.zeros(conv_step)), longdy=np.float64(1.0), longdydt=np.float64(1.0),
                 where_varies_most=J(np.zeros((nz, ni))), longdy_seen_min=np.float64(np.inf),
                 count_since_new_min=np.int32(0), rtol=np.float64(rtol), loss_criteria=np.float64(1e-3),
                 update_photo_frq=np.int32(1), is_final_photo_frq=np.bool_(False),
                 fix_species_started=np.bool_(False), fix_y=J(np.zeros((nz, ni))),
                 fix_mask=J(np.zeros((nz, ni), bool)), fix_pfix_idx=J(np.zeros(0, np.int32)),
                 h2he_pinned=np.bool_(False), h2he_mix=J(np.zeros(2)), y_evo=J(np.zeros((1, nz, ni))),
                 t_evo=J(np.zeros(1)), evo_idx=np.int32(0), chunk_target=np.int32(10 ** 6))
        f.update(over)
        return JS(**f)

    gas_all = np.ones(ni, bool)
    gas_part = gas_all.copy()
    gas_part[[2, 7]] = False
    y_neg = y0.copy()
    y_neg[4, 3] = -1e5
    y_small = y0.copy()
    y_small[[1, 5, 8], [6, 0, 11]] = -0.3
    rng = np.random.default_rng(61)
    fm = rng.random((nz, ni)) < 0.1
    cases = {
        # name: (y, rtol, dt, params, runner options, state overrides)
        "accept": (y0, 0.2, 1e-6, {}, {}, {}),
        "reject_delta": (y0, 1e-12, 1e-6, {}, {}, {}),
        "reject_loss": (y0, 0.2, 1e-6, dict(loss_eps=1e-300), {}, {}),
        "reject_nega": (y_neg, 0.2, 1e-6, {}, {}, {}),
        "force_retry": (y0, 1e-30, 1e-6, {}, {}, dict(retry_count=np.int32(8))),
        "force_underflow": (y0, 1e-30, 1.5e-14, {}, {}, {}),
        "gas_hydro": (y0, 0.2, 1e-6, dict(pos_cut=1e3), dict(non_gas=True, gas=gas_part, hydro_partial=True),
                      {}),
        "clip_small": (y_small, 0.2, 1e-6, dict(pos_cut=50.0), {}, {}),
        "fix": (y0, 0.2, 1e-6, dict(use_fix_species=True), {},
                dict(fix_mask=J(fm), fix_y=J(y0 * 1.01), fix_species_started=np.bool_(True))),
        "botrow_adapt": (y0, 0.2, 1e-6, dict(use_adapt_rtol=True), dict(zero_bot_row=True),
                         dict(accept_count=np.int32(10), loss_criteria=np.float64(1e-12))),
    }
    out = dict(net_text=np.array(case.net.text), k=case.k, compo=compo, atom_ini=atom_ini,
               case_names=np.array(list(cases) + ["chain"]))
    for kk in ATM_KEYS + FLAG_KEYS:
        out["atm_" + kk] = np.asarray(case.atm[kk])
    for k2, v in BODY_PARAMS.items():
        out["param_" + k2] = np.array(v)

    def run(name, y, rtol, dt, pover, ropt, sover, n_attempts=1):
        p = dict(BODY_PARAMS)
        p.update(pover)
        gas = ropt.get("gas", gas_all)
        runner = ns["_make_runner"](net, statics(p), ropt.get("non_gas", False), J(gas),
                                    ropt.get("zero_bot_row", False), J(np.zeros((nz, ni), bool)),
                                    ropt.get("hydro_partial", False), 1e30, 1e30)
        s = state(y, mix(np.abs(y), gas), dt, rtol, **sover)
        pre = {f: np.asarray(getattr(s, f)) for f in BODY_FIELDS}
        for kk, vv in pre.items():
            out[f"{name}_in_{kk}"] = vv
        for kk in ("fix_mask", "fix_y"):
            out[f"{name}_in_{kk}"] = np.asarray(getattr(s, kk))
        out[f"{name}_opt"] = np.array([float(pover.get("use_fix_species", False)),
                                       float(ropt.get("non_gas", False)), float(ropt.get("hydro_partial", False)),
                                       float(ropt.get("zero_bot_row", False)),
                                       float(pover.get("use_adapt_rtol", False)),
                                       float(p["loss_eps"]), float(p["pos_cut"])])
        out[f"{name}_gas"] = gas
        hist = []
        for _ in range(n_attempts):
            prev_acc, prev_retry = int(s.accept_count), int(s.retry_count)
            s = runner(s, atm)
            hist.append((int(s.accept_count) - prev_acc, int(s.retry_count), int(s.delta_count),
                         int(s.nega_count), int(s.loss_count)))
        for f_ in BODY_FIELDS:
            out[f"{name}_out_{f_}"] = np.asarray(getattr(s, f_))
        out[f"{name}_hist"] = np.array(hist, np.int64)
        print(f"body {name}: attempts {hist} dt {float(s.dt):.3e} delta {float(s.delta):.3e}")

    for name, (y, rtol, dt, pover, ropt, sover) in cases.items():
        run(name, y, rtol, dt, pover, ropt, sover)
    run("chain", y0, 1e-3, 3e-5, {}, {}, {}, n_attempts=8)
    np.savez_compressed(os.path.join(HERE, "body.npz"), **out)
    print("body: ok")

    # convergence chain: ring buffer, longdy / longdydt, stall detector and the
    # loop condition cond_fn (outer_loop.py:614-713, 919-989), recorded after
    # every attempt of the reference body
    cond_log = []

    def while_once(cond, fn, init):
        res = fn(init)
        cond_log.append(bool(cond(res)))
        return res

    ns["jax"].lax.while_loop = while_once
    conv_over = dict(count_min=2, yconv_cri=0.3, yconv_min=1.0, slope_cri=1e30, conv_stall_window=3,
                     trun_min=0.0, flux_cri=0.1, st_factor=0.5, mtol_conv=1e-20)
    p = dict(BODY_PARAMS)
    p.update(conv_over)
    runner = ns["_make_runner"](net, statics(p), False, J(gas_all), False, J(np.zeros((nz, ni), bool)), False,
                                1e30, 1e30)
    s = state(y0, mix(y0), 1e-6, 0.05, accept_count=np.int32(0), delta_count=np.int32(0), nega_count=np.int32(0),
              loss_count=np.int32(0), t=np.float64(0.0))
    conv_fields = ["accept_count", "retry_count", "t", "dt", "longdy", "longdydt", "longdy_seen_min",
                   "count_since_new_min"]
    cv = dict(conv_in_y=np.asarray(s.y), conv_in_ymix=np.asarray(s.ymix), conv_in_atom_loss=np.asarray(s.atom_loss),
              conv_n=np.array(40), conv_slope_min=np.array(1e-8))
    for k2, v in conv_over.items():
        cv["conv_param_" + k2] = np.array(v)
    rec = {f: [] for f in conv_fields}
    for _ in range(40):
        s = runner(s, atm)
        for f_ in conv_fields:
            rec[f_].append(np.asarray(getattr(s, f_)))
    for f_ in conv_fields:
        cv["conv_" + f_] = np.array(rec[f_])
    cv["conv_cond"] = np.array(cond_log)
    cv["conv_y_ring"] = np.asarray(s.y_time_ring)
    cv["conv_t_ring"] = np.asarray(s.t_time_ring)
    cv["conv_y"] = np.asarray(s.y)
    np.savez_compressed(os.path.join(HERE, "conv.npz"), **cv)
    print("conv: accepts", [int(a) for a in rec["accept_count"]], "cond", cond_log)


def photo_fixture(mods, syn):
    photo = mods["photo"]
    net = syn.make_network(21, 16, 40, n_photo=6)
    atm, extra = syn.make_atmosphere(21, net, nz=10)
    bins, din12 = syn.make_bins(2.0, 42.0, 0.25, 1.0, 22.0)
    ph = syn.make_photo(21, net, atm["Tco"], bins, din12, dbin1=0.25, dbin2=1.0, n_T_abs=1)
    pd = photo.PhotoData(absp_idx=ph["absp_idx"], absp_cross=ph["absp_cross"],
                         absp_T_idx=ph["absp_T_idx"], absp_T_cross=ph["absp_T_cross"],
                         scat_idx=ph["scat_idx"], scat_cross=ph["scat_cross"])
    y, dz, ymix = extra["y"], extra["dz"], extra["ymix"]
    tau = np.asarray(photo.compute_tau_jax(y, dz, pd))
    rng = np.random.default_rng(5)
    prev = np.abs(rng.normal(0, 1, tau.shape)) * 1e3
    res = {}
    for ag0 in (0.0, 0.3):
        aflux, sflux, dd, du = photo.compute_flux_jax(tau, ph["sflux_top"], ymix, pd, bins,
                                                      ph["mu_zenith"], ph["edd"], ag0, ph["hc"], prev,
                                                      ag0_is_zero=(ag0 == 0.0))
        tag = "ag0" if ag0 == 0.0 else "ag3"
        res.update({f"{tag}_aflux": np.asarray(aflux), f"{tag}_sflux": np.asarray(sflux),
                    f"{tag}_dflux_d": np.asarray(dd), f"{tag}_dflux_u": np.asarray(du)})
    Jb, JbT = photo.compute_J_jax_flat(res["ag0_aflux"], ph["cross_J"], ph["cross_J_T"],
                                       ph["din12_indx"], ph["dbin1"], ph["dbin2"])
    k = syn.make_rates(21, net, 10)
    act = np.ones(len(ph["branch_re_idx"]), bool)
    act[0] = False
    actT = np.ones(len(ph["branch_T_re_idx"]), bool)
    import _jax_numpy_shim as shim
    k_new = photo.update_k_with_J(k.view(shim.JArr), Jb, JbT, ph["branch_re_idx"], act, ph["branch_T_re_idx"], actT,
                                  0.5)
    save = dict(y=y, dz=dz, ymix=ymix, tau=tau, dflux_u_prev=prev, J_br=np.asarray(Jb),
                J_br_T=np.asarray(JbT), k=k, k_new=np.asarray(k_new), active=act, active_T=actT)
    save.update(res)
    for key, v in ph.items():
        save["ph_" + key] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, "photo.npz"), **save)
    print("photo: ok", tau.shape)


def chain_problem(mods):
    """The open chain 0 -> A -> B -> 0 of reference tests/test_steady_state_grad.py:44-132."""
    chem, jax_step = mods["chem"], mods["jax_step"]
    ni, nr, PAD, T = 2, 6, 2, 1
    r_idx = np.full((nr + 1, T), PAD, dtype=np.int64)
    p_idx = np.full((nr + 1, T), PAD, dtype=np.int64)
    r_st = np.zeros((nr + 1, T))
    p_st = np.zeros((nr + 1, T))
    p_idx[1, 0], p_st[1, 0] = 0, 1.0
    r_idx[3, 0], r_st[3, 0], p_idx[3, 0], p_st[3, 0] = 0, 1.0, 1, 1.0
    r_idx[5, 0], r_st[5, 0] = 1, 1.0
    three = np.zeros(nr + 1, dtype=bool)
    net = chem.NetworkArrays(ni=ni, nr=nr, reactant_idx=r_idx, product_idx=p_idx, reactant_stoich=r_st,
                             product_stoich=p_st, is_three_body=three)
    nz = 4
    atm = dict(Kzz=np.full(nz - 1, 1e-2), Dzz=np.full((nz - 1, ni), 1e-3), dzi=np.full(nz - 1, 1.0),
               vz=np.zeros(nz - 1), Hpi=np.full(nz - 1, 1.0), Ti=np.full(nz - 1, 1500.0), Tco=np.full(nz, 1500.0),
               g=np.full(nz, 1.0), ms=np.full(ni, 1.0), alpha=np.zeros(ni), M=np.full(nz, 1.0),
               vm=np.zeros((nz, ni)), vs=np.zeros((nz - 1, ni)), top_flux=np.zeros(ni), bot_flux=np.zeros(ni),
               bot_vdep=np.zeros(ni), gas_indx_mask=np.ones(ni, dtype=bool), use_vm_mol=False,
               use_settling=False, use_topflux=False, use_botflux=False)
    k = np.zeros((nr + 1, nz))
    k[1], k[3], k[5] = 1.0, 0.5, 0.3
    y0 = np.zeros((nz, ni))
    y0[:, 0], y0[:, 1] = 2.0, 3.3
    tables = dict(r_idx=r_idx, p_idx=p_idx, r_st=r_st, p_st=p_st, three=three)
    return net, atm, k, y0, tables


def adjoint_fixture(mods, syn):
    """Reference _ss_bwd (steady_state_grad.py:306-327) through the stand-in
    (its jax.vjp of chem_rhs in k is exact: chem_rhs is linear in k)."""
    import _jax_numpy_shim as shim
    ssg, solver = mods["steady_state_grad"], mods["solver"]
    out = {}
    net, atm_d, k, y0, tab = chain_problem(mods)
    atm = ref_atm(mods, atm_d)
    y = y0.copy()
    for it in range(100):
        r = np.asarray(ssg.steady_state_residual(y.view(shim.JArr), k.view(shim.JArr), atm, net))
        if np.max(np.abs(r)) < 1e-9:
            break
        diag, sup, sub = ssg._build_jacobian_blocks(y.view(shim.JArr), k.view(shim.JArr), atm, net)
        y = y + np.asarray(solver.block_thomas_diag_offdiag(diag, sup, sub, -r))
    v = np.zeros_like(y)
    v[:, 1] = 2.0 * y[:, 1]                       # d/dy of sum(y[:,1]**2)
    gk, _ = ssg._ss_bwd(atm, net, (k.view(shim.JArr), y.view(shim.JArr)), v.view(shim.JArr))
    out.update(chain_y=y, chain_v=v, chain_gk=np.asarray(gk), chain_newton_iters=np.array(it))
    for key, val in tab.items():
        out["chain_" + key] = val
    case = syn.make_case(seed=12, ni=12, n_fwd=30, nz=10, mild=True, k_range=(-40.0, 4.0), moldiff=True,
                         fluxes=True, n_three_body=6)
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(case.net.text)
        path = f.name
    rn = mods["network"].parse_network(path)
    os.unlink(path)
    netc = mods["chem"].to_jax(rn)
    atmc = ref_atm(mods, case.atm)
    v2 = np.random.default_rng(12).normal(0.0, 1.0, case.y.shape) / np.abs(case.y)
    gk2, _ = ssg._ss_bwd(atmc, netc, (case.k.view(shim.JArr), case.y.view(shim.JArr)), v2.view(shim.JArr))
    out.update(case_net_text=np.array(case.net.text), case_y=case.y, case_k=case.k, case_v=v2,
               case_gk=np.asarray(gk2))
    for kk in ATM_KEYS + FLAG_KEYS:
        out["case_atm_" + kk] = np.asarray(case.atm[kk])
    np.savez_compressed(os.path.join(HERE, "adjoint.npz"), **out)
    print("adjoint: ok, chain Newton iterations", it)


RATE_T = np.array([150.0, 180.0, 199.99, 200.0, 250.0, 277.5, 277.6, 300.0, 300.1, 420.0, 650.0, 800.0,
                   999.9, 1000.0, 1000.1, 1300.0, 1700.0, 2100.0, 2600.0, 3000.0])


def rates_fixture(mods, syn):
    """Reference rates.py / gibbs.py (plain NumPy, imported unmodified) on a
    seeded network with every rate form and seeded NASA-9 coefficients:
    forward constants, low-T caps, g/RT, K_eq, reverse fill, removal, the
    end-to-end build_rate_array, and the parser's rate columns and flags."""
    rates, gibbs = importlib.import_module("rates"), importlib.import_module("gibbs")
    text = syn.make_rate_network(0)
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(text)
        path = f.name
    rn = mods["network"].parse_network(path)
    os.unlink(path)
    coeffs = syn.make_nasa9(0, rn.ni)
    T = RATE_T
    M = 10.0 ** np.linspace(19.0, 10.0, T.shape[0])
    remove = [3, 8, 101, 250]
    k_fwd = rates.compute_forward_k(rn, T, M)
    k_caps = rates.apply_lowT_caps(rn, k_fwd, T, M)
    g = gibbs.gibbs_sp_vector(coeffs, T)
    K = gibbs.K_eq_array(rn, g, T)
    k_nocap = gibbs.fill_reverse_k(rn, k_fwd, K, remove_list=None)
    cfg = types.SimpleNamespace(use_lowT_limit_rates=True, remove_list=remove)
    atm = types.SimpleNamespace(Tco=T, M=M)
    k_all = rates.build_rate_array(cfg, rn, atm, coeffs)
    out = dict(net_text=np.array(text), coeffs=coeffs, T=T, M=M, remove=np.array(remove), k_fwd=k_fwd,
               k_caps=k_caps, g=g, K=K, k_nocap=k_nocap, k_all=k_all, stop_rev_indx=np.array(rn.stop_rev_indx))
    for f in ("a", "n", "E", "a_inf", "n_inf", "E_inf", "is_forward", "has_kinf", "is_special", "is_conden",
              "is_radiative", "is_photo", "is_ion"):
        out["net_" + f] = np.asarray(getattr(rn, f))
    np.savez_compressed(os.path.join(HERE, "rates.npz"), **out)
    print("rates: ok", k_all.shape, "nonzero", int((k_all != 0).sum()))


def refresh_fixture(mods):
    """Reference atm_refresh.py (update_mu_dz_jax with a reference layer
    inside the column, update_phi_esc_jax with the flux floor active for one
    species) and conden.py (update_conden_rates, apply_h2o_relax_jax,
    apply_nh3_relax_jax with condensing and evaporating layers) through the
    stand-in, on seeded inputs."""
    import _jax_numpy_shim as shim
    ar, cd = importlib.import_module("atm_refresh"), importlib.import_module("conden")
    rng = np.random.default_rng(21)
    nz, ni = 16, 12
    J = lambda a: np.asarray(a, dtype=np.float64).view(shim.JArr)  # noqa: E731
    ymix = 10.0 ** rng.uniform(-8, 0, (nz, ni))
    ymix /= ymix.sum(axis=1, keepdims=True)
    Tco = np.linspace(1800.0, 700.0, nz)
    pico = np.logspace(8.0, 0.0, nz + 1)
    n_0 = 0.5 * (pico[:-1] + pico[1:]) / (1.380649e-16 * Tco)
    y = ymix * n_0[:, None]
    mol_mass = rng.uniform(2.0, 60.0, ni)
    ms = mol_mass / 6.02214076e23
    Dzz_top = 10.0 ** rng.uniform(5.0, 9.0, ni)
    esc = np.array([0, 3, 7], dtype=np.int32)
    kb, Navo, gs, Rp = 1.38064852e-16, 6.02214086e23, 2140.0, 7.1492e9
    top_flux = rng.normal(0.0, 1e6, ni)
    pref = 5
    max_flux = float(np.sort(np.abs(Dzz_top[esc] * y[-1, esc] / 1e7))[1])   # floors one of the three
    st = ar.AtmRefreshStatic(Tco=J(Tco), pico=J(pico), mol_mass=J(mol_mass), ms=J(ms), Dzz_top=J(Dzz_top),
                             diff_esc_idx=esc, pref_indx=pref, zco_pref=0.0, gs=gs, Rp=Rp, kb=kb, Navo=Navo,
                             max_flux=max_flux, nz=nz, ni=ni)
    mu, g, Hp, dz, zco, dzi, Hpi = (np.asarray(v) for v in ar.update_mu_dz_jax(J(ymix), st))
    tf = np.asarray(ar.update_phi_esc_jax(J(y), J(g), J(Hp), J(top_flux), st))
    # condensation: two condensing species (H2O-like at 1, NH3-like at 4) with condensates 2 and 5
    nr = 20
    k = 10.0 ** rng.uniform(-20, -10, (nr + 1, nz))
    re_idx = np.array([11, 15], dtype=np.int32)
    sp_idx = np.array([1, 4], dtype=np.int32)
    Dg = 10.0 ** rng.uniform(-2, 1, (2, nz))
    sat_n = y[:, sp_idx].T * rng.uniform(0.5, 1.5, (2, nz))
    coeff = np.array([3.0e-9, 0.0])
    gas = np.ones(ni, dtype=bool)
    gas[[2, 5]] = False
    h2o_Dg, nh3_Dg = Dg[0], Dg[1]
    h2o_sat, nh3_sat = sat_n[0], sat_n[1]
    y[:, 2] = y[:, 1] * rng.uniform(0.0, 0.5, nz)
    y[:, 5] = y[:, 4] * rng.uniform(0.0, 0.5, nz)
    dt = 3.0e4
    cst = cd.CondenStatic(conden_re_idx=re_idx, conden_sp_idx=sp_idx, Dg_per_re=J(Dg), sat_n_per_re=J(sat_n),
                          coeff_per_re=J(coeff), h2o_active=True, h2o_idx=1, h2o_l_s_idx=2, h2o_Dg=J(h2o_Dg),
                          h2o_sat=J(h2o_sat), h2o_m_over_rho_r2=0.7, nh3_active=True, nh3_idx=4, nh3_l_s_idx=5,
                          nh3_Dg=J(nh3_Dg), nh3_sat=J(nh3_sat), nh3_m_over_rho_r2=0.3, nh3_conden_top=9,
                          n_0=J(n_0), gas_indx_mask=gas)
    k_new = np.asarray(cd.update_conden_rates(J(k), J(y), cst))
    y1, x1 = cd.apply_h2o_relax_jax(J(y), J(ymix), dt, cst)
    y2, x2 = cd.apply_nh3_relax_jax(y1, x1, dt, cst)
    out = dict(ymix=ymix, Tco=Tco, pico=pico, mol_mass=mol_mass, ms=ms, Dzz_top=Dzz_top, esc=esc, pref=np.array(pref),
               consts=np.array([kb, Navo, gs, Rp, max_flux]), top_flux=top_flux, y=y, n_0=n_0, mu=mu, g=g, Hp=Hp,
               dz=dz, zco=zco, dzi=dzi, Hpi=Hpi, top_flux_new=tf, k=k, re_idx=re_idx, sp_idx=sp_idx, Dg=Dg,
               sat_n=sat_n, coeff=coeff, gas=gas, dt=np.array(dt), k_new=k_new, y_h2o=np.asarray(y1),
               ymix_h2o=np.asarray(x1), y_nh3=np.asarray(y2), ymix_nh3=np.asarray(x2))
    np.savez_compressed(os.path.join(HERE, "refresh.npz"), **out)
    tau_h2o = 1.0 / (h2o_Dg * 0.7 * (y[:, 1] - h2o_sat))
    print("refresh: ok; h2o condensing layers", int((tau_h2o > 0).sum()), "of", nz)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("VULCAN_REFERENCE"),
                    required="VULCAN_REFERENCE" not in os.environ,
                    help="the reference checkout (default: $VULCAN_REFERENCE)")
    ap.add_argument("--only", default="", help="comma-separated fixture names (default: all)")
    args = ap.parse_args()
    mods, shim = load_reference(args.reference)
    syn = importlib.import_module("jax-vulcan_b200.synthetic")
    only = set(filter(None, args.only.split(",")))
    if only:
        for name in sorted(only):
            if name == "body":
                body_fixture(mods, syn, args.reference, shim)
            elif name == "rates":
                rates_fixture(mods, syn)
            elif name == "refresh":
                refresh_fixture(mods)
            else:
                raise SystemExit(f"--only supports: body, rates, refresh (got {name})")
        return
    mild = dict(mild=True, k_range=(-40.0, 4.0))
    step_fixture(mods, "plain", syn.make_case(seed=5, ni=12, n_fwd=30, nz=10, **mild), n_steps=3)
    step_fixture(mods, "moldiff", syn.make_case(seed=6, ni=12, n_fwd=30, nz=10, moldiff=True, **mild))
    step_fixture(mods, "full", syn.make_case(seed=7, ni=12, n_fwd=30, nz=12, moldiff=True,
                                             advection=True, fluxes=True, n_three_body=8, **mild))
    case = syn.make_case(seed=8, ni=12, n_fwd=30, nz=10, moldiff=True, fluxes=True, **mild)
    fm = np.random.default_rng(8).random(case.y.shape) < 0.1
    step_fixture(mods, "fixmask", case, fix_mask=fm)
    step_fixture(mods, "medium", syn.make_case(seed=9, ni=30, n_fwd=185, nz=24, moldiff=True,
                                               n_three_body=20, **mild))
    # spec-like stiff draw (k log-uniform over [1e-45, 1e-6], dt = 1e-6): an
    # ill-conditioned step; only its chemistry RHS/Jacobian are compared elementwise.
    step_fixture(mods, "stiff", syn.make_case(seed=10, ni=30, n_fwd=185, nz=24, k_range=(-45.0, -6.0),
                                              n_three_body=20))
    thomas_fixture(mods)
    contract_fixture(mods)
    photo_fixture(mods, syn)
    adjoint_fixture(mods, syn)
    body_fixture(mods, syn, args.reference, shim)
    rates_fixture(mods, syn)
    refresh_fixture(mods)


if __name__ == "__main__":
    main()
