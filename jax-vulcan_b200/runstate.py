"""The device loop carry as the reference's ``RunState`` runner slots
(reference `state.py:106-160`, `:187-209`).

``runstate_slots`` gives, for one atmosphere of a batched ``LoopState``, the
four runner-state slots of the reference pytree as dicts with its field
names - ``step`` (StepInputs: y, y_prev, ymix, t, dt, longdy, longdydt,
y_evo, t_evo), ``params`` (ParamInputs), ``atoms`` (AtomInputs) and, with
photochemistry, ``photo_runtime`` (PhotoRuntimeInputs) - as host NumPy
values. ``state_from_runstate`` rebuilds a batched device carry from such
slots (one per atmosphere); the runner-internal values the reference pytree
does not carry (retry count, the adaptive rtol, the loss criterion, the stall
record) start from the reference's pre-loop values, as its runner does when it
starts from a RunState. The static slots (atm, rate, photo, metadata) belong
to the reference's configuration and atmosphere setup and are not restated.
"""
from __future__ import annotations

import numpy as np

STEP_FIELDS = ("y", "y_prev", "ymix", "t", "dt", "longdy", "longdydt", "y_evo", "t_evo")
PARAM_FIELDS = ("count", "nega_count", "loss_count", "delta_count", "delta", "small_y", "nega_y", "end_case",
                "switch_final_photo_frq", "pic_count", "where_varies_most", "fix_species_start")
ATOM_FIELDS = ("atom_order", "atom_ini", "atom_loss", "atom_loss_prev", "atom_sum")
PHOTO_FIELDS = ("tau", "aflux", "sflux", "dflux_d", "dflux_u", "prev_aflux", "aflux_change")


def runstate_slots(state, b, compo, atom_order, atom_ini, photo_carry=None):
    """Runner-state slots of atmosphere ``b`` of ``state`` (a ``LoopState``;
    its convergence record, when enabled, gives longdy, longdydt, end_case and
    the photo-frequency switch). ``compo`` [ni, n_atoms], ``atom_ini``
    [n_atoms] or [B, n_atoms]; ``photo_carry``: ``photo.PhotoCarry``."""
    snap = state.snapshot()
    rec = {k: np.asarray(v).reshape(-1)[b] for k, v in snap.items() if np.ndim(v) == 1}
    y = snap["y"][b]
    conv = state.conv_host()[b] if state.conv is not None else None
    ai = np.asarray(atom_ini, np.float64)
    ai = ai[b] if ai.ndim == 2 else ai
    step = dict(y=y.copy(), y_prev=snap["y_prev"][b].copy(), ymix=snap["ymix"][b].copy(), t=float(rec["t"]),
                dt=float(snap["dt"][b]), longdy=float(conv["longdy"]) if conv is not None else 1.0,
                longdydt=float(conv["longdydt"]) if conv is not None else 1.0,
                y_evo=np.zeros((0, 0, 0)), t_evo=np.zeros((0,)))
    params = dict(count=int(rec["accept_count"]), nega_count=int(rec["nega_count"]),
                  loss_count=int(rec["loss_count"]), delta_count=int(rec["delta_count"]), delta=float(rec["delta"]),
                  small_y=float(rec["small_y"]), nega_y=float(rec["nega_y"]),
                  end_case=1 if (conv is not None and int(conv["done"])) else 0,
                  switch_final_photo_frq=bool(conv["is_final_photo_frq"]) if conv is not None else False,
                  pic_count=0, where_varies_most=np.zeros_like(y), fix_species_start=False)
    atoms = dict(atom_order=tuple(atom_order), atom_ini=ai.copy(), atom_loss=snap["atom_loss"][b].copy(),
                 atom_loss_prev=snap["atom_loss_prev"][b].copy(),
                 atom_sum=np.einsum("zi,ia->a", y, np.asarray(compo, np.float64)))
    out = dict(step=step, params=params, atoms=atoms, photo_runtime=None)
    if photo_carry is not None:
        h = lambda t: t[b].detach().cpu().numpy().copy()  # noqa: E731
        out["photo_runtime"] = dict(tau=h(photo_carry.tau), aflux=h(photo_carry.aflux), sflux=h(photo_carry.sflux),
                                    dflux_d=h(photo_carry.dflux_d), dflux_u=h(photo_carry.dflux_u),
                                    prev_aflux=h(photo_carry.aflux),
                                    aflux_change=float(conv["aflux_change"]) if conv is not None else 0.0)
    return out


def state_from_runstate(slots, rtol=0.2, loss_criteria=1e-3, conv_step=None, update_photo_frq=0):
    """A batched device ``LoopState`` from per-atmosphere runner slots (a list
    of ``runstate_slots`` dicts). ``conv_step``: enable the convergence
    carry with longdy / longdydt from the slots (the stall record restarts,
    as at the start of the reference runner)."""
    from .outer_loop import LoopState
    st = [s["step"] for s in slots]
    pa = [s["params"] for s in slots]
    at = [s["atoms"] for s in slots]
    stack = lambda rows, f: np.stack([np.asarray(r[f], np.float64) for r in rows])  # noqa: E731
    counters = {"accept_count": np.array([p["count"] for p in pa]), "nega_count": np.array([p["nega_count"] for p in pa]),
                "loss_count": np.array([p["loss_count"] for p in pa]),
                "delta_count": np.array([p["delta_count"] for p in pa])}
    state = LoopState(stack(st, "y"), stack(st, "ymix"), np.array([s["dt"] for s in st]), stack(at, "atom_loss"),
                      stack(at, "atom_loss_prev"), y_prev=stack(st, "y_prev"), t=np.array([s["t"] for s in st]),
                      rtol=rtol, loss_criteria=loss_criteria, counters=counters,
                      small_y=np.array([p["small_y"] for p in pa]), nega_y=np.array([p["nega_y"] for p in pa]))
    rec = state.scalars_host().copy()
    rec["delta"] = [p["delta"] for p in pa]
    import torch
    state.scalars = torch.from_numpy(rec.view(np.uint8).copy()).cuda()
    if conv_step is not None:
        state.enable_convergence(conv_step, update_photo_frq=update_photo_frq)
        from .outer_loop import CONV_DTYPE
        c = state.conv_host().copy()
        c["longdy"] = [s["longdy"] for s in st]
        c["longdydt"] = [s["longdydt"] for s in st]
        c["is_final_photo_frq"] = [int(p["switch_final_photo_frq"]) for p in pa]
        state.conv = torch.from_numpy(c.view(np.uint8).copy()).cuda()
        assert c.dtype == CONV_DTYPE
    return state
