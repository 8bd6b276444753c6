"""Host logic of Simulation.minimize's FP32 stall rule (no GPU): the chunk statistics that
end an FP32 phase when the arrested flow can no longer build velocity."""
import numpy as np

from soliton_solver_b200.core.simulation import fp32_stalled


def _alternating(E0, n, amp, drift):
    """A free step lowers E by amp, the next (arrested) step raises it by amp - drift."""
    E = [E0]
    for k in range(n):
        E.append(E[-1] - amp if k % 2 == 0 else E[-1] + amp - drift)
    return np.array(E[1:])


def test_strict_alternation_with_a_small_energy_change_is_a_stall():
    E = _alternating(8.6, 1000, 1e-9, 1e-12)
    assert fp32_stalled(8.6, E, 1e-9)


def test_two_consecutive_decreases_mean_the_flow_still_moves():
    E = _alternating(8.6, 1000, 1e-9, 1e-12)
    E[501:] -= 2e-9  # step 501 lowers the energy again right after the free step 500
    assert not fp32_stalled(8.6, E, 1e-9)


def test_a_rising_saddle_flow_is_not_a_stall():
    E = 635.0 + 1e-9 * np.arange(1, 1001)  # E rises on every step while the flow converges
    assert not fp32_stalled(635.0, E, 1e-9)


def test_alternation_with_a_large_energy_change_is_not_a_stall():
    E = _alternating(8.6, 1000, 1e-6, 1e-7)  # 5e-5 lower over the chunk
    assert not fp32_stalled(8.6, E, 1e-9)


def test_short_chunks_are_never_stalls():
    assert not fp32_stalled(1.0, np.array([1.0]), 1e-9)
