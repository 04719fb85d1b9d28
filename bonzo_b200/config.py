"""config.cfg reader with the reference's lookup semantics.

Mirrors ``read_param(section, key, dtype, usr_dir)`` of src/io/read_config.pyx:10-38
(Python 3 ``configparser`` in place of the Python 2 ``ConfigParser`` the
reference imports).  Keys are looked up by the spelling the reference's code
reads; where the example config.cfg uses another spelling (e.g. ``Lx`` for
``xmax``, ``hst_dt`` for ``history_dt``) that alias is accepted too, the
code's spelling winning when both are present.
"""
import configparser
import os

# key the code reads -> spellings seen in the shipped config.cfg
ALIASES = {
    ("computation", "xmax"): ["Lx"],
    ("computation", "ymax"): ["Ly"],
    ("computation", "zmax"): ["Lz"],
    ("output", "history_dt"): ["hst_dt"],
    ("output", "slice_dt"): ["slc_dt"],
    ("output", "variable_type"): ["var_type"],
    ("output", "write_ghost_cells"): ["write_ghost"],
    ("restart", "restart_dt"): ["rst_dt"],
    ("physics", "f0"): ["f"],
    ("physics", "nmod"): ["Nmod"],
}

# defaults for keys that the reference's shipped config.cfg does not carry
DEFAULTS = {
    ("computation", "xmin"): 0.0,
    ("computation", "ymin"): 0.0,
    ("computation", "zmin"): 0.0,
    ("computation", "xmax"): 1.0,
    ("computation", "ymax"): 1.0,
    ("computation", "zmax"): 1.0,
    ("computation", "x_scale"): "uni",
    ("computation", "y_scale"): "uni",
    ("computation", "z_scale"): "uni",
    ("computation", "limiter"): "vl",
    ("computation", "charact_proj"): 0,
    ("computation", "tintegr"): "vl",
    ("computation", "cour_diff"): 0.5,
    ("physics", "geometry"): "car",
    ("physics", "kappa0"): 0.0,
    ("physics", "elec_thcond_type"): "aniso",
    ("physics", "sat_hfe"): 0,
}


class ConfigError(ValueError):
    pass


def _parser(usr_dir):
    path = os.path.join(usr_dir, "config.cfg")
    if not os.path.exists(path):
        raise ConfigError("cannot read parameters: unable to open the input file %s" % path)
    cp = configparser.ConfigParser(inline_comment_prefixes=("#",))
    cp.optionxform = str  # keys are case sensitive in the reference (Nx, Lx, ...)
    cp.read(path)
    return cp


def read_param(section, key, dtype, usr_dir, default=None):
    """read_config.pyx:10-38: dtype 'f' float, 'i' int, 's' string."""
    cp = _parser(usr_dir)
    names = [key] + ALIASES.get((section, key), [])
    for name in names:
        if cp.has_option(section, name):
            raw = cp.get(section, name).strip()
            try:
                if dtype == "f":
                    return float(raw)
                if dtype == "i":
                    return int(float(raw))
                return raw
            except ValueError as e:
                raise ConfigError("bad value for [%s] %s: %r" % (section, name, raw)) from e
    if default is not None:
        return default
    if (section, key) in DEFAULTS:
        return DEFAULTS[(section, key)]
    raise ConfigError("missing parameter [%s] %s in %s/config.cfg" % (section, key, usr_dir))


def read_user_param(key, dtype, usr_dir, default=None):
    """Problem-generator parameters live in the [problem] section."""
    return read_param("problem", key, dtype, usr_dir, default)
