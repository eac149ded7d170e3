"""Host compilation of elements into the flat table: flags the kernels act on."""
import numpy as np

from at_b200 import elements as E
from at_b200 import table as T
from at_b200.lattice import compile_lattice
from conftest import ELECTRON_REST


def _flags(cl):
    hdr = cl.words.view(np.uint64)
    return [(int(hdr[int(o)]) >> T.ATB_H_FL_SHIFT) & T.ATB_H_FL_MASK for o in cl.offsets[:-1]]


def test_upright_flag_marks_multipoles_without_skew_terms():
    line = [E.Quadrupole("Q", 0.5, 1.2),
            E.Multipole("S", 0.2, [0.0, 0.0, 0.1], [0.0, 0.0, 5.0]),
            E.Multipole("K", 0.2, [0.0, 0.0], [0.0, 1.0], KickAngle=np.array([0.0, 1e-4])),
            E.Multipole("Z", 0.2, [-0.0, 0.0], [0.0, 1.0])]
    flags = _flags(compile_lattice(line, 3e9, ELECTRON_REST))
    assert flags[0] & T.ATB_F_NOSKEW            # upright quadrupole
    assert not flags[1] & T.ATB_F_NOSKEW        # skew sextupole component
    assert not flags[2] & T.ATB_F_NOSKEW        # vertical KickAngle folds into A[0]
    assert flags[3] & T.ATB_F_NOSKEW            # a signed zero is zero
