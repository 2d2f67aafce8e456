"""CPU oracle for the adaptive-step caller contract of the reference runner.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``smoke()`` and the CPU
baseline of ``bench.py``; never by the product path.

Restates, from reference `outer_loop.py`:

* ``atom_loss``      -> `_compute_atom_loss` (`:171-178`)
* ``step_size``      -> `_step_size` (`:181-193`)
* ``clip``           -> `_make_clip_fn` (`:196-224`)
* ``aggregate_delta`` -> `_make_aggregate_delta_fn` (`:227-250`)
* ``controller_step`` -> the accept / force-accept / time / dt logic of
  `body_fn` (`:733-768`, `:1031-1038`) for a run without photo, condensation,
  atmosphere refresh or adaptive rtol.
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


def controller_step(state, k, atm, net, compo, atom_ini, p):
    """One attempt of the adaptive loop. ``state``: dict(y, ymix, dt, t,
    atom_loss_prev, retry). ``p``: rtol, atol, mtol, pos_cut, nega_cut,
    loss_eps, dt_var_min, dt_var_max, dt_min, dt_max, max_retries.
    Returns the new state dict plus ``accept``, ``force``, ``delta``."""
    y, dt = state["y"], state["dt"]
    sol, delta_arr = ros2.ros2_step(y, k, dt, atm, net)
    sol_c, ymix_new, _, _ = clip(sol, state["ymix"], p["mtol"], p["pos_cut"], p["nega_cut"])
    al = atom_loss(sol_c, compo, atom_ini)
    delta = aggregate_delta(sol_c, delta_arr, state["ymix"], p["mtol"], p["atol"])
    accept = bool(np.all(sol_c >= 0) and np.max(np.abs(al - state["atom_loss_prev"])) < p["loss_eps"]
                  and delta <= p["rtol"])
    next_reject = dt * p["dt_var_min"]
    force = (not accept) and (next_reject < p["dt_min"] or state["retry"] >= p["max_retries"])
    do_acc = accept or force
    t_next = state["t"] + (p["dt_min"] if force else dt) if do_acc else state["t"]
    dt_norm = step_size(dt, delta, p["rtol"], p["dt_var_min"], p["dt_var_max"], p["dt_min"], p["dt_max"])
    dt_force = step_size(p["dt_min"], delta, p["rtol"], p["dt_var_min"], p["dt_var_max"], p["dt_min"], p["dt_max"])
    dt_next = dt_force if force else (dt_norm if accept else next_reject)
    out = dict(state)
    if do_acc:
        out.update(y=sol_c, ymix=ymix_new, atom_loss_prev=al, retry=0)
    else:
        out.update(retry=state["retry"] + 1)
    out.update(t=t_next, dt=float(dt_next), accept=accept, force=force, delta=float(delta))
    return out
