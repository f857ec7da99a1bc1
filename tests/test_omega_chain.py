"""The size of the one deliberate departure from the reference's Bingham
collision, measured on the oracle (CPU, no GPU needed).

C6 relaxes each node with OMEGA_MRT as the previous node of its sweep left
it (C6:890 reads, C6:958 writes): a serial chain that shifts the viscosity
field by one node along x.  The GPU relaxes each node with its own omega of
the previous step (oracle rule omega_chain=0).  On the C6 program at 40 x
150 (L_C = 10) over 3000 steps:

  yield number 0.066 (the disk creeps through a mostly unyielded fluid):
  the terminal v_y of the two rules differ by about 26 % and about 1.6 % of
  the fluid nodes carry a different yield flag at the end.  The difference
  is the chain's one-node shift of the yield surface: it is about 15 % at
  L_C = 20 and 3 % at L_C = 40 (tests/golden/omega_chain_study.py).
  yield number 0.5 (the disk is held by the yield stress): below 0.1 %, no
  flag differs.

The bounds below pin those measurements, so a change of either rule shows.
"""

import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import omega_chain_study as ocs  # noqa: E402


def _departure(y, nx=40, ny=150, steps=3000):
    r1 = ocs.run((nx, ny, y, steps, 1))
    r0 = ocs.run((nx, ny, y, steps, 0))
    _, disk = ocs.case(nx, ny, y)
    return ocs.compare({1: r1[0], 0: r0[0]}, {1: r1[1], 0: r0[1]}, {1: r1[2], 0: r0[2]},
                       disk[0, 1])


def test_omega_rule_departure_creeping_disk():
    m = _departure(0.066)
    assert m["vy_chain"] < 0 and m["vy_own"] < 0
    assert 0.15 <= m["vy_rel_diff"] <= 0.35, m
    assert m["flag_diff_frac"] <= 0.03, m


def test_omega_rule_departure_held_disk():
    m = _departure(0.5)
    assert m["vy_rel_diff"] <= 2e-3, m
    assert m["flag_diff_frac"] == 0.0, m
    assert m["unyielded_frac"] == pytest.approx(1.0)
