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
