"""GPU tests of LOCDYN_W_MatrixMarket / LOCDYN_Dump on a device-assembled
local dynamics (b2gs_locdyn_w_matrix_market, b2gs_locdyn_dump): the text
equals the restatement oracle/ldy_formats.py on the oracle's assembly of the
same scene with the same R, U, character for character (the device assembly
is bitwise the oracle's)."""
import numpy as np
import pytest

import oracle
import ldy_formats
from solfec_b200 import LOCDYN
from test_formats_cpu import cases, spatial_points

pytestmark = pytest.mark.gpu


def test_device_formats(tmp_path):
    rng = np.random.default_rng(2)
    for k, sc in enumerate(cases()):
        ld = oracle.assemble(sc)
        n = ld.n
        R, U = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
        ldy = LOCDYN()
        ldy.update_begin(sc)
        ldy.set_state(R, U)
        p = str(tmp_path / ('w%d.mtx' % k))
        ldy.w_matrix_market(p)
        assert open(p).read() == ldy_formats.matrix_market(n, ld.W, ld.adjptr, ld.adjcol, ld.Woff)
        pts = spatial_points(sc)
        p = str(tmp_path / ('d%d.txt' % k))
        ldy.dump(p, pts, sc.master, sc.slave, sc.base)
        assert open(p).read() == ldy_formats.dump(n, pts, sc.master, sc.slave, sc.base, ld.W, ld.B, ld.V, U, R,
                                                   ld.adjptr, ld.adjcol, ld.Woff)
        ldy.close()
