"""Number format of the solver files written by the library (C++ restatement of Java's
Double.toString, fp_java_double): the documented Java strings and agreement with the Python
writer of the optimisation export on seeded doubles of every magnitude (CPU; no GPU call)."""
import struct

import numpy as np
import pytest

import flowpro_v2_b200 as fg
from flowpro_v2_b200 import optexport
from tests.test_optexport import JAVA_STRINGS


@pytest.mark.parametrize("x,s", JAVA_STRINGS)
def test_library_java_double_format(x, s):
    assert fg.java_double(x) == s


def test_library_java_double_matches_export_writer_and_reads_back():
    rng = np.random.default_rng(11)
    xs = list(rng.standard_normal(3000) * 10.0 ** rng.integers(-15, 15, 3000))
    xs += [struct.unpack("<d", struct.pack("<Q", int(b)))[0] for b in rng.integers(0, 2 ** 63, 3000, dtype=np.uint64)]
    for x in xs:
        s = fg.java_double(x)
        assert s == optexport.java_double(x)
        if np.isfinite(x):
            assert float(s.replace("E", "e")) == x
