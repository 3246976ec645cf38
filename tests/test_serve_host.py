"""Host logic of the serving loop that needs no GPU: how many steps a tick
takes under a frame interval (matter_tests_b200.serve.Server._tick_steps)."""
import numpy as np

from matter_tests_b200.serve import Server


def _server(frame_ms, samples):
    srv = Server(budget_bytes=1, tick_steps=8, frame_ms=frame_ms)
    for p, t in samples:
        srv._fit.append((p, t))
    return srv


def test_fixed_ticks_without_a_frame_interval():
    srv = _server(None, [(p, 0.2 + 1e-6 * p) for p in (1e4, 1e5, 1e6, 4e6)])
    assert srv._tick_steps(1e7) == 8


def test_one_step_ticks_until_the_model_has_four_samples():
    srv = _server(8.0, [(p, 0.2 + 1e-6 * p) for p in (1e4, 1e5, 1e6)])
    assert srv._tick_steps(1e3) == 1 and srv._tick_steps(1e7) == 1


def test_steps_fit_the_frame_on_a_linear_step_time():
    # 0.2 ms + 1 ms per million particles per step
    srv = _server(8.0, [(p, 0.2 + 1e-6 * p) for p in (1e4, 1e5, 5e5, 1e6, 4e6)])
    assert srv._tick_steps(1e6) == 6        # 8 / 1.2
    assert srv._tick_steps(3.7e6) == 2      # 8 / 3.9
    assert srv._tick_steps(5e7) == 1        # one step even when it overruns the frame
    assert srv._tick_steps(1e3) == 8        # never more than tick_steps


def test_one_batch_size_falls_back_to_a_proportional_model():
    srv = _server(8.0, [(1e6, 2.0)] * 6)
    assert srv._tick_steps(1e6) == 4
    assert srv._tick_steps(4e6) == 1
    assert 1 <= srv._tick_steps(2e5) <= 8


def test_noisy_samples_still_give_steps_in_range():
    rng = np.random.default_rng(3)
    P = rng.uniform(1e4, 5e6, 64)
    srv = _server(16.0, [(p, (0.3 + 1e-6 * p) * rng.uniform(0.8, 1.3)) for p in P])
    for p in (1e3, 1e5, 1e6, 1e7, 1e8):
        assert 1 <= srv._tick_steps(p) <= 8
    assert srv._tick_steps(1e8) == 1 and srv._tick_steps(1e3) == 8
