"""The raw binary dump format of the mini-app's diagnostics
(mom6_diag.F90:362-431) and the number format of its statistics line
(post_data's '(A,A,A,4ES14.6)'), as hackathon_mom6_miniapp_b200.diag_format
reads and writes them.  No GPU needed."""
import numpy as np

from hackathon_mom6_miniapp_b200.diag_format import (dump_name, es14_6, read_bin,
                                                      stats_line, write_bin)


def test_2d_round_trip_and_layout(tmp_path):
    a = np.arange(12, dtype=np.float64).reshape(4, 3, order="F") * 0.5
    p = tmp_path / "f.bin"
    write_bin(p, a)
    raw = p.read_bytes()
    assert len(raw) == 8 + 8 * 12
    assert np.frombuffer(raw[:8], dtype="<i4").tolist() == [4, 3]
    # values in column-major order: a(1,1), a(2,1), ...
    assert np.frombuffer(raw[8:], dtype="<f8").tolist() == a.flatten(order="F").tolist()
    b = read_bin(p)
    assert b.shape == (4, 3) and np.array_equal(a, b)


def test_3d_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    a = np.asfortranarray(rng.normal(size=(5, 4, 3)))
    p = tmp_path / "g.bin"
    write_bin(p, a)
    raw = p.read_bytes()
    assert len(raw) == 12 + 8 * 60
    assert np.frombuffer(raw[:12], dtype="<i4").tolist() == [5, 4, 3]
    assert np.array_equal(read_bin(p), a)


def test_es14_6():
    assert es14_6(0.0) == "  0.000000E+00"
    assert es14_6(1.0) == "  1.000000E+00"
    assert es14_6(-1.5e-7) == " -1.500000E-07"
    assert es14_6(123456.789) == "  1.234568E+05"
    # three-digit exponents lose the letter (ESw.d with the default exponent width)
    assert es14_6(1.7976931348623157e308) == "  1.797693+308"
    assert es14_6(-2.5e-100) == " -2.500000-100"
    assert all(len(es14_6(x)) == 14 for x in (0.0, -1e300, 3.3, -7e-5))


def test_stats_line_and_file_names():
    assert stats_line("KE", (0.0, 1.0, 0.5, 0.25)) == (
        "  Diag: KE min/max/mean/rms:   0.000000E+00  1.000000E+00  5.000000E-01  2.500000E-01")
    assert dump_name("./", "mass", 8) == ".//mass000008.bin"
    assert dump_name("/tmp/x", "diffu_sum", 123456) == "/tmp/x/diffu_sum123456.bin"
    assert dump_name("d", "KE", 1234567) == "d/KE******.bin"
