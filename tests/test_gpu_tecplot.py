"""amrlbm_write_tecplot (TecPlot_CellCenter, TecPlot_ASCII.f90:2-86) through the
C ABI: the file the library writes from the device state equals, byte for
byte, the file tests/tecplot_ref.py restates from the oracle's state after the
same steps; an unwritable path is reported as AMRLBM_ERR_IO."""
import pytest

import amrlbm
from amrlbm import AmrLbm, AmrLbmError
from oracle_lib import Oracle
from tecplot_ref import tecplot_text

pytestmark = pytest.mark.gpu

CASES = {"reference_default": amrlbm.reference_params, "small_16x16": amrlbm.workload_small}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("steps", [0, 3])
def test_tecplot_file_matches_the_restated_writer(case, steps, tmp_path):
    p = CASES[case]()
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    if steps:
        orc.main_loop(steps)
    path = tmp_path / "Rising_Bubble_2D_00.dat"
    with AmrLbm(p) as gpu:
        gpu.initialize_rising_bubble()
        if steps:
            gpu.main_loop(steps)
        gpu.sync()
        gpu.tecplot_cell_center(str(path), steps)
    assert path.read_text() == tecplot_text(orc, p, steps)


def test_unwritable_path_is_reported(tmp_path):
    with AmrLbm(amrlbm.reference_params()) as gpu:
        gpu.initialize_rising_bubble()
        with pytest.raises(AmrLbmError) as e:
            gpu.tecplot_cell_center(str(tmp_path / "no_such_dir" / "out.dat"), 0)
        assert e.value.status == amrlbm.ERR_IO
