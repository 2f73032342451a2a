"""CPU tests of the drivers' output records: turbdata.out lines printed as the
HIT driver's ofstream (precision 17, a space after each value) prints them,
and the cylinder driver's raw-double records (time, then the values)."""
import numpy as np

import mpi_3dcompact_b200 as m


def test_turbdata_line_format(tmp_path):
    p = tmp_path / "turbdata.out"
    vals = [0.0, 1.0 / 3.0, 1e-5, 123456.789, -2.5e-300, 7.0, 0.1, 1e20, 2.0 ** -30, 3.0, 42.0]
    m.append_turbdata_line(p, vals)
    m.append_turbdata_line(p, vals[::-1])
    lines = p.read_text().split("\n")
    assert lines[-1] == "" and len(lines) == 3
    for line, want in zip(lines[:2], (vals, vals[::-1])):
        assert line.endswith(" ")
        toks = line[:-1].split(" ")
        # std::ostream with precision(17) and no floatfield prints as %.17g
        assert toks == ["%.17g" % v for v in want]
        assert [float(t) for t in toks] == want


def test_cylinder_record_layout(tmp_path):
    p = tmp_path / "cylinderP.dat"
    a, b = np.linspace(0.0, 1.0, 7), np.arange(7.0)
    m.append_record(p, 0.25, a)
    m.append_record(p, 0.5, b)
    raw = np.fromfile(p, dtype=np.float64)
    assert raw.size == 2 * 8
    assert raw[0] == 0.25 and np.array_equal(raw[1:8], a)
    assert raw[8] == 0.5 and np.array_equal(raw[9:], b)
