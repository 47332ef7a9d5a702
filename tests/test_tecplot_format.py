"""The Fortran edit descriptors of TecPlot_CellCenter (TecPlot_ASCII.f90:78-84)
as restated in tests/tecplot_ref.py, against known Fortran results, and the
restated file's structure on the oracle's start-up state (CPU only)."""
import amrlbm
from oracle_lib import Oracle
from tecplot_ref import fortran_e, fortran_f, fortran_i, records, tecplot_text


def test_e14_6_known_answers():
    assert fortran_e(1.0) == "  0.100000E+01"
    assert fortran_e(-1.0) == " -0.100000E+01"
    assert fortran_e(0.0) == "  0.000000E+00"
    assert fortran_e(-0.0) == " -0.000000E+00"
    assert fortran_e(-0.000123456789) == " -0.123457E-03"
    assert fortran_e(9.9999996) == "  0.100000E+02"   # rounding carries into the exponent
    assert fortran_e(0.5) == "  0.500000E+00"
    assert fortran_e(1e-100) == "  0.100000E-99"
    assert fortran_e(1e-101) == "  0.100000-100"     # three exponent digits drop the E
    assert fortran_e(-2.5e200) == " -0.250000+201"


def test_f10_3_and_iw_known_answers():
    assert fortran_f(0.5) == "     0.500"
    assert fortran_f(12.3456) == "    12.346"
    assert fortran_f(0.0) == "     0.000"
    assert fortran_f(1.0e9) == "**********"
    assert fortran_i(123, 7) == "    123"
    assert fortran_i(999999, 6) == "999999"
    assert fortran_i(1000000, 6) == "******"


def test_format_reversion():
    assert records(["a", "b", "c"], 2) == "ab\nc\n"
    assert records(["a", "b"], 2) == "ab\n"
    assert records([], 9) == ""


def test_restated_file_structure_on_the_startup_state():
    p = amrlbm.reference_params()
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    text = tecplot_text(orc, p, 0)
    lines = text.split("\n")
    nleaf = len(orc.leaves())
    nn, ne = nleaf * (p.nx + 1) * (p.ny + 1), nleaf * p.nx * p.ny
    assert lines[0] == " Variables = X, Y, Ux, Uy, C, P"
    assert lines[1] == f"Zone N ={nn:6d}, E ={ne:6d}, ZONETYPE=FEquadrilateral, DATAPACKING=Block"
    assert lines[2] == ' VARLOCATION=([3,4,6]=CELLCENTERED), T = "0"'
    ceil = lambda a, b: -(-a // b)
    expect = 3 + 2 * ceil(nn, 9) + 2 * ceil(ne, 8) + ceil(nn, 9) + ceil(ne, 8) + ceil(4 * ne, 8)
    assert len(lines) == expect + 1 and lines[-1] == ""
    # node C at the start-up: -1/2 .. 1/2
    first_c = 3 + 2 * ceil(nn, 9) + 2 * ceil(ne, 8)
    vals = [float(lines[first_c][k:k + 14]) for k in range(0, 14 * 9, 14)]
    assert all(-0.5 - 1e-12 <= x <= 0.5 + 1e-12 for x in vals)
