"""CPU oracle for the adaptive-step caller contract of the reference runner.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``smoke()`` and the CPU
baseline of ``bench.py``; never by the product path.

Restates, from reference `outer_loop.py`:

* ``atom_loss``      -> `_compute_atom_loss` (`:171-178`)
* ``step_size``      -> `_step_size` (`:181-193`)
* ``clip``           -> `_make_clip_fn` (`:196-224`)
* ``aggregate_delta`` -> `_make_aggregate_delta_fn` (`:227-250`)
* ``body_update`` / ``attempt`` -> the state update of one attempt of
  `body_fn` (`:715-1100`): accept / reject / force-accept, hydrostatic
  rebalance, counters, adaptive rtol and dt, for a run without photo,
  condensation, atmosphere refresh, ion balance or bottom pins.
* ``conv_update`` / ``loop_continues`` -> the convergence ring and
  diagnostics (`:633-670`, `:918-989`) and `cond_fn` (`:672-713`)
* ``photo_switch`` / ``photo_due`` -> the photo-frequency switch
  (`:1040-1050`) and the photo cadence (`:716-724`)
"""
from __future__ import annotations

import numpy as np

from . import ros2


def atom_loss(y, compo, atom_ini):
    return (np.einsum("zi,ia->a", y, compo) - atom_ini) / atom_ini


def step_size(dt, delta, rtol, dt_var_min, dt_var_max, dt_min, dt_max):
    delta_eff = np.where(delta == 0.0, 0.01 * rtol, delta)
    h = 0.9 * (rtol / delta_eff) ** 0.5
    h = np.clip(h, dt_var_min, dt_var_max)
    return np.clip(dt * h, dt_min, dt_max)


def clip(y_in, ymix_old, mtol, pos_cut, nega_cut, gas_mask=None):
    small = np.sum(np.where((y_in < pos_cut) & (y_in >= 0), np.abs(y_in), 0.0))
    nega = np.sum(np.where((y_in > nega_cut) & (y_in <= 0), np.abs(y_in), 0.0))
    y = np.where((y_in < pos_cut) & (y_in >= nega_cut), 0.0, y_in)
    y = np.where((ymix_old < mtol) & (y < 0), 0.0, y)
    if gas_mask is not None:
        ysum = np.sum(np.where(np.asarray(gas_mask, bool)[None, :], y, 0.0), axis=1, keepdims=True)
    else:
        ysum = np.sum(y, axis=1, keepdims=True)
    return y, y / ysum, small, nega


def aggregate_delta(sol, delta_arr, ymix_old, mtol, atol, zero_bot_row=False, cond_zero=None):
    m = np.where(ymix_old < mtol, 0.0, delta_arr)
    m = np.where(sol < atol, 0.0, m)
    if zero_bot_row:
        m = m.copy()
        m[0] = 0.0
    if cond_zero is not None:
        m = np.where(np.asarray(cond_zero, bool), 0.0, m)
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = np.where(sol > 0, m / np.maximum(np.abs(sol), 1e-300), 0.0)
    return np.max(ratio)


BODY_FIELDS = ["y", "y_prev", "ymix", "dt", "t", "delta", "accept_count", "retry_count", "atom_loss",
               "atom_loss_prev", "nega_count", "loss_count", "delta_count", "small_y", "nega_y", "rtol",
               "loss_criteria"]


def mix_from_y(y, gas=None):
    """`_mix_from_y` (`outer_loop.py:593-600`): y / ysum over gas species (all without a mask)."""
    if gas is None:
        return y / np.sum(y, axis=1, keepdims=True)
    return y / np.sum(np.where(np.asarray(gas, bool)[None, :], y, 0.0), axis=1, keepdims=True)


def body_update(s, sol, delta_arr, M, compo, atom_ini, p, gas=None, hydro_partial=False,
                zero_bot_row=False, fix_mask=None, fix_y=None, conden=None, cond_zero=None):
    """State after one attempt of the reference loop body given the step's
    (sol, delta_arr): fixed species (`outer_loop.py:733-739`), clip, atom loss,
    error norm (`:741-743`), accept / force-accept (`:745-756`), reject
    counters (`:758-764`), time (`:766-768`), hydrostatic rebalance
    (`:844-853`), next y / ymix / atom loss (`:899-914`), counters
    (`:916-917`, `:1062-1066`), adaptive rtol (`:990-1020`) and dt
    (`:1022-1031`). Photo, condensation, atmosphere refresh, ion balance,
    bottom pins, the convergence ring and save_evolution are not restated.

    ``s``: dict with ``BODY_FIELDS``; ``p``: loss_eps, pos_cut, nega_cut, mtol,
    atol, dt_var_min, dt_var_max, dt_min, dt_max, batch_max_retries,
    use_adapt_rtol, rtol_min, rtol_max, adapt_rtol_dec_period,
    adapt_rtol_inc_period, adapt_rtol_dec, adapt_rtol_inc, adapt_rtol_loss_mul,
    adapt_rtol_inc_loss_thresh. ``gas``: gas-species mask when non-gas species
    are present (the ysum of clip and mix), else None. ``cond_zero``: species
    mask [ni] whose delta the error norm drops (`:244`), or None.
    """
    if fix_mask is not None:
        sol = np.where(fix_mask, fix_y, sol)
        delta_arr = np.where(fix_mask, 0.0, delta_arr)
    sol_clip, ymix_new, small_inc, nega_inc = clip(sol, s["ymix"], p["mtol"], p["pos_cut"], p["nega_cut"], gas)
    al_new = atom_loss(sol_clip, compo, atom_ini)
    cz = None if cond_zero is None else np.broadcast_to(np.asarray(cond_zero, bool)[None, :], sol_clip.shape)
    delta = aggregate_delta(sol_clip, delta_arr, s["ymix"], p["mtol"], p["atol"], zero_bot_row, cz)
    rtol = s["rtol"]
    loss_diff = np.max(np.abs(al_new - s["atom_loss_prev"]))
    accept = bool(np.all(sol_clip >= 0) & (loss_diff < p["loss_eps"]) & (delta <= rtol))
    next_reject = s["dt"] * p["dt_var_min"]
    force = bool((next_reject < p["dt_min"]) | (s["retry_count"] >= p["batch_max_retries"])) and not accept
    do_acc = accept or force
    reject = not do_acc
    too_big = bool(delta > rtol)
    any_neg = bool(np.any(sol_clip < 0))
    t_next = s["t"] + (p["dt_min"] if force else s["dt"]) if do_acc else s["t"]

    # condensation (outer_loop.py:770-800): on a taken attempt inside the time
    # window, ``conden(sol_clip, ymix_new, dt)`` (the relaxation of
    # conden.py:74-160 with the attempt's dt) replaces the clipped state
    # before the hydrostatic rebalance; the caller rewrites the condensation
    # rows of k from the clipped state before it (``_sol_clip_raw``)
    sol_clip_raw, fired = sol_clip, False
    if conden is not None and do_acc and s["t"] >= conden["start_time"]:
        sol_clip, ymix_new = conden["fn"](sol_clip, ymix_new, s["dt"])
        fired = True

    bal_full = M[:, None] * ymix_new
    if hydro_partial:
        bal = np.where(np.asarray(gas, bool)[None, :], bal_full, sol_clip)
    else:
        bal = bal_full
    ymix_bal = mix_from_y(bal, gas)
    al_bal = atom_loss(bal, compo, atom_ini)
    if force:
        y_next, ymix_next, al_next = np.where(s["y_prev"] < 0, 0.0, s["y_prev"]), s["ymix"], s["atom_loss_prev"]
    elif accept:
        y_next, ymix_next, al_next = bal, ymix_bal, al_bal
    else:
        y_next, ymix_next, al_next = s["y_prev"], s["ymix"], s["atom_loss"]

    out = dict(s)
    out.update(y=y_next, ymix=ymix_next, atom_loss=al_next, t=t_next, delta=delta)
    if do_acc:
        out.update(y_prev=y_next, atom_loss_prev=al_next, accept_count=s["accept_count"] + 1, retry_count=0,
                   small_y=s["small_y"] + small_inc, nega_y=s["nega_y"] + nega_inc)
    else:
        out.update(retry_count=s["retry_count"] + 1)
    out.update(delta_count=s["delta_count"] + int(reject and too_big),
               nega_count=s["nega_count"] + int(reject and not too_big and any_neg),
               loss_count=s["loss_count"] + int(reject and not too_big and not any_neg))

    lc = s["loss_criteria"]
    if p["use_adapt_rtol"] and do_acc:
        max_loss = np.max(np.abs(al_new))
        acc = s["accept_count"]
        if acc % p["adapt_rtol_dec_period"] == 0 and max_loss >= lc:
            rtol = max(rtol * p["adapt_rtol_dec"], p["rtol_min"])
            lc = lc * p["adapt_rtol_loss_mul"]
        if acc % p["adapt_rtol_inc_period"] == 0 and acc > 0 and max_loss < p["adapt_rtol_inc_loss_thresh"]:
            rtol = min(rtol * p["adapt_rtol_inc"], p["rtol_max"])
    dt_norm = step_size(s["dt"], delta, rtol, p["dt_var_min"], p["dt_var_max"], p["dt_min"], p["dt_max"])
    dt_force = step_size(p["dt_min"], delta, rtol, p["dt_var_min"], p["dt_var_max"], p["dt_min"], p["dt_max"])
    out.update(dt=float(dt_force if force else (dt_norm if accept else next_reject)), rtol=rtol, loss_criteria=lc)
    out["_accept"], out["_force"] = accept, force
    out["_sol_clip"], out["_ymix_new"] = sol_clip, ymix_new   # the refresh's inputs (outer_loop.py:818-826)
    out["_sol_clip_raw"], out["_conden_fired"] = sol_clip_raw, fired
    return out


def attempt(s, k, atm, net, compo, atom_ini, p, **kw):
    """One attempt: the Ros2 step from ``s["y"]`` then ``body_update``."""
    sol, delta_arr = ros2.ros2_step(s["y"], k, s["dt"], atm, net, fix_mask=kw.get("fix_mask"))
    return body_update(s, sol, delta_arr, atm["M"], compo, atom_ini, p, **kw)


CONV_FIELDS = ["longdy", "longdydt", "longdy_seen_min", "count_since_new_min"]


def conv_update(s, ring_y, ring_t, n_0, p, ignore=None, do_accept=True):
    """Ring append and convergence diagnostics after one attempt (the state
    ``s`` is the post-attempt state: y, ymix, t, accept_count and the carried
    longdy fields). Follows `outer_loop.py:918-928` (ring slot
    ``max(accept_count - 1, 0) % conv_step`` rewritten with (y, t)),
    `_conv_jax` `:633-670` (lookback to the ring entry nearest ``t *
    st_factor``, the newest slot excluded; longdy = max over the masked
    relative change), `:944-989` (longdy / longdydt kept only on accept; the
    stall counter restarts on a 5 % drop). ``p``: conv_step, st_factor,
    mtol_conv, atol. Rings are updated in place; returns the new fields."""
    conv = p["conv_step"]
    acc = int(s["accept_count"])
    idx = max(acc - 1, 0) % conv
    ring_y[idx] = s["y"]
    ring_t[idx] = s["t"]
    diffs = np.abs(ring_t - s["t"] * p["st_factor"])
    diffs[idx] = np.inf
    k = int(np.argmin(diffs))
    la = np.abs((s["y"] - ring_y[k]) / n_0[:, None])
    la = np.where(s["ymix"] < p["mtol_conv"], 0.0, la)
    la = np.where(s["y"] < p["atol"], 0.0, la)
    if ignore is not None:
        la = np.where(np.asarray(ignore, bool)[None, :], 0.0, la)
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = np.where(s["ymix"] > 0, la / np.maximum(s["ymix"], 1e-300), 0.0)
    ld_new = np.max(ratio)
    ldt_new = ld_new / max(s["t"] - ring_t[k], 1e-300)
    out = {}
    out["longdy"] = ld_new if do_accept else s["longdy"]
    out["longdydt"] = ldt_new if do_accept else s["longdydt"]
    drop = do_accept and out["longdy"] < s["longdy_seen_min"] * 0.95
    out["longdy_seen_min"] = out["longdy"] if drop else s["longdy_seen_min"]
    out["count_since_new_min"] = 0 if drop else (s["count_since_new_min"] + 1 if do_accept else
                                                 s["count_since_new_min"])
    return out


def loop_continues(s, p, slope_min, aflux_change=0.0):
    """`cond_fn` (`outer_loop.py:672-713`) without the chunk cap: False once the
    run is too long, has too many accepted steps, or is ready and converged
    (or stalled). ``p``: runtime, count_max, trun_min, count_min, yconv_cri,
    slope_cri, yconv_min, flux_cri, conv_stall_window."""
    too_long = s["t"] > p["runtime"]
    too_many = s["accept_count"] > p["count_max"]
    conv = (((s["longdy"] < p["yconv_cri"]) and (s["longdydt"] < p["slope_cri"]))
            or ((s["longdy"] < p["yconv_min"]) and (s["longdydt"] < slope_min)))
    conv = conv and aflux_change < p["flux_cri"]
    stalled = (s["count_since_new_min"] > p["conv_stall_window"] and s["longdy_seen_min"] < p["yconv_min"]
               and s["longdy"] < p["yconv_min"] and aflux_change < p["flux_cri"])
    ready = s["t"] > p["trun_min"] and s["accept_count"] > p["count_min"]
    return not (too_long or too_many or (ready and (conv or stalled)))


def photo_switch(s, p):
    """Photo-frequency switch from the initial to the final cadence once
    longdy and longdydt (after this attempt's update) drop below their
    thresholds (reference `outer_loop.py:1040-1050`). ``p``: use_photo,
    photo_switch_longdy, photo_switch_longdydt, final_update_photo_frq."""
    sw = (bool(p["use_photo"]) and not s["is_final_photo_frq"] and s["longdy"] < p["photo_switch_longdy"]
          and s["longdydt"] < p["photo_switch_longdydt"])
    return dict(update_photo_frq=p["final_update_photo_frq"] if sw else s["update_photo_frq"],
                is_final_photo_frq=bool(s["is_final_photo_frq"] or sw))


def photo_due(s, p):
    """Whether the next attempt runs the photo branch: no retry pending and
    ``accept_count % update_photo_frq == 0`` (reference `outer_loop.py:716-724`)."""
    return bool(p["use_photo"]) and s["retry_count"] == 0 and s["accept_count"] % s["update_photo_frq"] == 0
