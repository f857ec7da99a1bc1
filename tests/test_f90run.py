"""Known answers for the Fortran-subset translator that produces the golden
fixtures (tests/golden/f90run.py): literal kinds, mixed-kind promotion,
integer division, powers, SUM order, derived types, value-result arguments
and static locals."""

import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import f90run  # noqa: E402

SRC = """
MODULE PARAM
  DOUBLE PRECISION,PARAMETER :: W(0:2)=(/4.0/9.0,1.0/9.0,1.0/36.0/)
  INTEGER,PARAMETER :: N=3
  TYPE REC
    DOUBLE PRECISION :: X(1:2)
    DOUBLE PRECISION :: M
  END TYPE
END MODULE PARAM
PROGRAM T
  USE PARAM
  IMPLICIT NONE
  DOUBLE PRECISION :: A,B,C,S(1:4),Q
  REAL :: R
  INTEGER :: I,J,K
  TYPE(REC) :: P(1:2)
  A=0.05; B=0.05D0; R=1.0/3.0; C=1.0/3.0
  I=-7/2; J=MOD(-7,2); K=2**10
  S=(/1.0D0,1.0D-16,1.0D-16,1.0D-16/)
  P%M=2.0
  P(2)%X=(/3.0D0,4.0D0/)
  Q=0.0
  CALL BUMP(Q); CALL BUMP(Q)
  WRITE(20,*) A,B,R,C,I,J,K,SUM(S),W(2),P(1)%M,P(2)%X(2),Q,(1.1D0)**3
  STOP
END
SUBROUTINE BUMP(X)
  IMPLICIT NONE
  DOUBLE PRECISION :: X, CNT=0.0
  CNT=CNT+1.0
  X=X+CNT
END SUBROUTINE BUMP
"""


def test_translator_semantics():
    frame, io, _ = f90run.run_program(SRC)
    (rec,) = io[20]
    a, b, r, c, i, j, k, s, w2, m, x22, q, cube = rec
    assert a == float(np.float32("0.05")) and a != 0.05      # default REAL literal
    assert b == 0.05                                          # D exponent
    assert r == float(np.float32(1.0) / np.float32(3.0))      # REAL(4) arithmetic
    assert c == r                                             # single division, then widened
    assert (i, j, k) == (-3, -1, 1024)                        # truncating division, MOD sign
    assert s == ((1.0 + 1e-16) + 1e-16) + 1e-16               # sequential SUM
    assert w2 == float(np.float32(1.0) / np.float32(36.0))
    assert m == 2.0 and x22 == 4.0                            # array-of-structure assignment
    assert q == 3.0                                           # value-result + static local (1 + 2)
    assert cube == (1.1 * 1.1) * 1.1                          # x**3 as (x*x)*x
