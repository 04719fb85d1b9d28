"""config.cfg lookup semantics (read_config.pyx:10-38) and host-side grid setup."""
import numpy as np
import pytest

from bonzo_b200.config import ConfigError, read_param
from bonzo_b200.coords import GridCoord


def write_cfg(tmp_path, text):
    (tmp_path / "config.cfg").write_text(text)
    return str(tmp_path)


def test_read_param_types_and_aliases(tmp_path):
    d = write_cfg(tmp_path, "[computation]\nNx: 64\nLx: 2.\ncour: 0.4  # CFL\nrsolver: hlld\n"
                            "[physics]\ngam: 1.66667\n")
    assert read_param("computation", "Nx", "i", d) == 64
    assert read_param("computation", "xmax", "f", d) == 2.0  # alias Lx
    assert read_param("computation", "cour", "f", d) == 0.4
    assert read_param("computation", "rsolver", "s", d) == "hlld"
    assert read_param("computation", "limiter", "s", d) == "vl"  # default (key absent)
    with pytest.raises(ConfigError):
        read_param("physics", "bc_x1", "i", d)


def test_code_spelling_wins(tmp_path):
    d = write_cfg(tmp_path, "[computation]\nxmax: 3.\nLx: 2.\n")
    assert read_param("computation", "xmax", "f", d) == 3.0


def test_missing_file(tmp_path):
    with pytest.raises(ConfigError):
        read_param("computation", "Nx", "i", str(tmp_path / "nope"))


def test_coordinates_periodic_ghosts():
    gc = GridCoord(96, 1, 1, dims=1, bc=((0, 0), (0, 0), (0, 0)), ng=3)
    assert gc.Ntot == [102, 1, 1]
    assert gc.i1 == 3 and gc.i2 == 98
    assert np.allclose(gc.dlf[0], 1 / 96, rtol=1e-12)
    assert gc.lf[0][gc.i1] == 0.0
    assert gc.lf[0][gc.i2 + 1] == 1.0
    assert np.allclose(gc.lf[0][:gc.i1], -np.arange(gc.i1, 0, -1) / 96, rtol=1e-12)


def test_oracle_and_host_coordinates_agree():
    from oracle.oracle import OracleSim
    for bc in (0, 1, 2):
        gc = GridCoord(48, 40, 1, dims=2, bc=((bc, bc), (bc, bc), (0, 0)), ng=3)
        s = OracleSim(48, 40, 1, dims=2, bc=((bc, bc), (bc, bc), (0, 0)))
        for ax in range(3):
            lf, lv, dlf = s.coords(ax)
            assert np.array_equal(lf, gc.lf[ax])
            assert np.array_equal(lv, gc.lv[ax])
            assert np.array_equal(dlf, gc.dlf[ax])
