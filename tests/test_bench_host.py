"""The reporting logic of bench.py's JFNK comparison on CPU, with the device solve replaced by
scripted results: every arm is timed `repeats` times and reports its fastest converged run,
all times are listed, the speed-ups are taken against block Jacobi's reported time, and the
other arms get 3x that time as their budget."""
import pytest

import bench


class FakeBody:
    n_points = 500_000


def scripted(monkeypatch, script):
    """Replace the device solve: script[arm] is the list of results of its successive runs."""
    calls = []
    left = {k: list(v) for k, v in script.items()}

    def arm(pd, mpnn, nkm, body, device, pc, G, increments, n_steps, weights, gmres_maxiter,
            newton_maxiter, budget):
        calls.append((pc, G, budget))
        r = left[pc].pop(0)
        return None if r is None else dict(r, group=G)
    monkeypatch.setattr(bench, "_jfnk_arm", arm)
    import pdcuda.train_preconditioner as tp
    monkeypatch.setattr(tp, "bending_beam", lambda *a, **k: FakeBody())
    return calls


def test_best_of_two_and_speedups(monkeypatch):
    calls = scripted(monkeypatch, {
        "block_jacobi": [{"s": 6.6, "gmres_iters": 8648}, {"s": 6.5, "gmres_iters": 8648}],
        "block_poly": [{"s": 3.0, "gmres_iters": 2848}, {"s": 3.1, "gmres_iters": 2848}],
        "learned_poly": [{"s": 3.9, "gmres_iters": 2570}, {"s": 2.8, "gmres_iters": 2570}],
    })
    res = bench.jfnk_compare(0, 2, repeats=2)
    arms = res["arms"]
    assert res["points"] == 500_000
    assert arms["block_jacobi"]["s"] == 6.5 and arms["block_jacobi"]["repeats_s"] == [6.6, 6.5]
    assert arms["block_poly"]["s"] == 3.0 and arms["block_poly"]["repeats_s"] == [3.0, 3.1]
    assert arms["learned_poly"]["s"] == 2.8 and arms["learned_poly"]["repeats_s"] == [3.9, 2.8]
    assert arms["block_jacobi"]["speedup_vs_block_jacobi"] == 1.0
    assert arms["learned_poly"]["speedup_vs_block_jacobi"] == pytest.approx(6.5 / 2.8)
    # block Jacobi runs without a budget; the others get 3x its reported time
    assert [b for pc, _, b in calls if pc == "block_jacobi"] == [None, None]
    assert all(b == pytest.approx(19.5) for pc, _, b in calls if pc != "block_jacobi")
    assert len(calls) == 6


def test_a_faster_unconverged_run_is_not_reported(monkeypatch):
    scripted(monkeypatch, {
        "block_jacobi": [{"s": 6.0}, {"s": 6.2}],
        "block_poly": [{"s": 1.0, "converged": False, "increments_done": 1}, {"s": 3.0}],
        "learned_poly": [None, {"s": 2.5}],
    })
    arms = bench.jfnk_compare(0, 2, repeats=2)["arms"]
    assert arms["block_poly"]["s"] == 3.0 and arms["block_poly"]["repeats_s"] == [1.0, 3.0]
    assert arms["block_poly"]["speedup_vs_block_jacobi"] == pytest.approx(2.0)
    assert arms["learned_poly"]["s"] == 2.5 and arms["learned_poly"]["repeats_s"] == [None, 2.5]


def test_single_run_lists_no_repeats(monkeypatch):
    scripted(monkeypatch, {"block_jacobi": [{"s": 6.0}], "block_poly": [{"s": 3.0}],
                           "learned_poly": [{"s": 2.0, "converged": False}]})
    arms = bench.jfnk_compare(0, 2)["arms"]
    assert "repeats_s" not in arms["block_jacobi"]
    # an arm that did not converge gets no speed-up
    assert "speedup_vs_block_jacobi" not in arms["learned_poly"]
