"""Stage sequence of the n_max continuation (lib_mie_ms_calculate_scattering_coefficients_ab_nm,
FoggySim/src/lib/mie_theory/lib_mie_multi_sphere.f90:162-371) with a fake solver on the CPU, and
the initial-guess embedding between degree ranges."""
import numpy as np

from itofoggysim_b200.solver import MultiSphereSolver, continuation_stages


def trace(n_org, n_start=None, step=None, dynamic=False, berr=lambda n, it: 1e-9):
    seq = []

    def run(n, it):
        seq.append((n, it))
        return berr(n, it)
    continuation_stages(run, n_org, n_start, step, dynamic)
    return seq


def test_plain_and_two_stage():
    assert trace(12) == [(12, None)]
    assert trace(12, 4) == [(4, 100), (12, 1000)]


def test_fixed_steps():
    # do n = n_start, n_org - step, step (Fortran bounds inclusive), then n_org
    assert trace(8, 2, 2) == [(2, 100), (4, 100), (6, 100), (8, 1000)]
    assert trace(9, 2, 3) == [(2, 100), (5, 100), (9, 1000)]
    assert trace(8, 7, 3) == [(8, 1000)]


def test_dynamic_accepted_steps_advance_twice():
    # every trial accepted: the degree moves by the step at the trial and again before the solve
    assert trace(12, 2, 4, True) == [(2, None), (6, 1), (10, 1000), (12, 1), (12, 1000)]


def test_dynamic_rejected_trial_halves_the_step():
    # trials at steps > 1 fail above degree 5: step 4 -> 2 -> 1, each retry from the degree tried
    seq = trace(12, 2, 4, True, berr=lambda n, it: 1.0 if (it == 1 and n > 5) else 1e-9)
    assert seq == [(2, None), (6, 1), (8, 1), (10, 1000), (12, 1), (12, 1), (12, 1000)]


def test_step_one_is_a_plain_march():
    assert trace(5, 2, 1, True) == [(2, None), (4, 1000), (5, 1000)]


def test_embed_between_degree_ranges():
    rng = np.random.default_rng(0)
    c3, c5 = 15, 35
    x = rng.standard_normal(2 * 2 * c3) + 1j * rng.standard_normal(2 * 2 * c3)
    up = MultiSphereSolver.embed(x, 2, 3, 5).reshape(2, 2, c5)
    assert np.array_equal(up[:, :, :c3], x.reshape(2, 2, c3)) and np.all(up[:, :, c3:] == 0)
    down = MultiSphereSolver.embed(up.reshape(-1), 2, 5, 3)
    assert np.array_equal(down, x)
