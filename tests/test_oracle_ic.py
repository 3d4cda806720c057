"""The oracle's seeded workload states (oracle/hype_oracle_ic.c) against the
library's generators (include/hype_ic.h): the same bits.

The CPU legs of bench.py (the CPU baseline and the reference arm) build their
inputs with the oracle's copy so they never load the library; this pin keeps
their inputs identical to the GPU arm's.
"""
import numpy as np
import pytest

import oracle as O

KAP = dict(gamma1=4.4, gamma2=1.4, pi1=6.0e8, pi2=0.0)
EUL = dict(gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0)


@pytest.mark.parametrize("nx,ny,seed,nb", [(67, 45, 0, 1), (128, 96, 3, 4), (5, 301, 11, 2), (256, 256, 0, 4)])
def test_shock_bubble_bits(hp, nx, ny, seed, nb):
    c = O.Config(system=O.KAPILA, nx=nx, ny=ny, **KAP)
    a = O.initial_state(c, "shock_bubble", seed=seed, nbubbles=nb)
    b = hp.initial_state(hp.Config(system=hp.KAPILA_5EQN, nx=nx, ny=ny, **KAP), "shock_bubble", seed=seed, nbubbles=nb)
    assert a.tobytes() == b.tobytes()


@pytest.mark.parametrize("nx,ny,seed", [(64, 64, 0), (97, 33, 5), (200, 150, 7)])
def test_bn_discs_bits(hp, nx, ny, seed):
    c = O.Config(system=O.BN, nx=nx, ny=ny, **KAP)
    a = O.initial_state(c, "bn_discs", seed=seed)
    b = hp.initial_state(hp.Config(system=hp.BAER_NUNZIATO, nx=nx, ny=ny, **KAP), "bn_discs", seed=seed)
    assert a.tobytes() == b.tobytes()


@pytest.mark.parametrize("nx,ny,seed", [(64, 64, 0), (33, 71, 9)])
def test_euler_quadrants_bits(hp, nx, ny, seed):
    c = O.Config(system=O.EULER, nx=nx, ny=ny, x_min=-1.0, x_max=1.0, y_min=-1.0, y_max=1.0, **EUL)
    a = O.initial_state(c, "euler_quadrants", seed=seed)
    b = hp.initial_state(hp.Config(system=hp.EULER, nx=nx, ny=ny, x_min=-1.0, x_max=1.0, y_min=-1.0, y_max=1.0, **EUL),
                         "euler_quadrants", seed=seed)
    assert a.tobytes() == b.tobytes()


def test_kind_must_fit_system():
    with pytest.raises(ValueError):
        O.initial_state(O.Config(system=O.BN, nx=8, ny=8), "shock_bubble")
