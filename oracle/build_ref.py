"""Build the reference's own C kernels into oracle/_ref/ (test infrastructure).

Reads the C sources of the reference where they lie: the directory given as
the first argument, else $BNZ_REF_ROOT, else a checkout named `reference`
beside this repository (../reference relative to the repository root).  It
compiles patched copies in a temporary directory outside
the repository (deleted afterwards), and writes ONLY the shared libraries
under oracle/_ref/ (git-ignored; they travel to the GPU box).

The reference does not compile as shipped.  Four one-line compile fixes are
applied to the copies (the reference's defect list D5-D8):
  D5  src/defs_c.h:128-129,142-143   FMAX/FMIN macros take two arguments
  D6  src/coordinates/coord_c.h:49   missing ';' after `int interp_order`
  D7  src/coordinates/reconstr_c.c:44-47  `(gc->geom)[ax]` on a scalar
  D8  src/mhd/eos_c.c:61-63,84-86    unbraced loop bodies in prim2char_1 /
                                     char2prim_1
D23 src/mhd/eos_c.h:445 (hydro build only) loop bound BX exists only with
    MFIELD,
and D9 (non-static inline definitions in eos_c.h emitted by every TU) is
handled at link time with --allow-multiple-definition.

Outputs:
  oracle/_ref/libbnzref.so        MFIELD=1 (hll, hllt, hlld, eos, reconstr)
  oracle/_ref/libbnzref_hydro.so  MFIELD=0 (hll, hllc, hllt, eos, reconstr)
"""
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
FILES = [
    "src/defs_c.h",
    "src/mhd/eos_c.c",
    "src/mhd/eos_c.h",
    "src/mhd/fluxes_c.c",
    "src/mhd/fluxes_c.h",
    "src/coordinates/reconstr_c.c",
    "src/coordinates/reconstr_c.h",
    "src/coordinates/coord_c.h",
]
CFLAGS = ["-std=gnu99", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
          "-DSPREC=0", "-w"]


def _patch(rel, text):
    if rel == "src/defs_c.h":
        text = re.sub(r"#define FMAX\(a\) \( fmax(f?)\(a\) \)",
                      r"#define FMAX(a,b) ( fmax\1(a,b) )", text)
        text = re.sub(r"#define FMIN\(a\) \( fmin(f?)\(a\) \)",
                      r"#define FMIN(a,b) ( fmin\1(a,b) )", text)
    elif rel == "src/coordinates/coord_c.h":
        text = re.sub(r"int interp_order(\s*)//", r"int interp_order;\1//", text)
    elif rel == "src/coordinates/reconstr_c.c":
        text = re.sub(r"\(gc->geom\s*\)\[ax\]", "(gc->geom)", text)
    elif rel == "src/mhd/eos_c.h":
        # D23 (hydro builds only): primcons2flux bounds its loop by BX, which
        # exists only with MFIELD; hydro builds use the full NMODE.
        text = text.replace(
            "  for (int n=0; n<BX; ++n)\n",
            "#if MFIELD\n  for (int n=0; n<BX; ++n)\n#else\n  for (int n=0; n<NMODE; ++n)\n#endif\n")
    elif rel == "src/mhd/eos_c.c":
        text = re.sub(
            r"for \(int n=0; n<NMODE; \+\+n\)\n(\s*)w\[n\] = w1\[n\]\[i\];\n\s*vc\[n\] = vc1\[n\]\[i\];",
            r"for (int n=0; n<NMODE; ++n) {\n\1w[n] = w1[n][i];\n\1vc[n] = vc1[n][i]; }",
            text)
    return text


# a reference checkout beside the repository, found relative to this file
DEFAULT_REF_ROOT = os.path.normpath(os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..",
                                                 "reference"))


def build(ref_root=None, quiet=False):
    ref_root = ref_root or os.environ.get("BNZ_REF_ROOT") or DEFAULT_REF_ROOT
    if not os.path.isdir(os.path.join(ref_root, "src", "mhd")):
        if not quiet:
            print("build_ref: reference sources not found at %s; skipped" % ref_root)
        return False
    os.makedirs(OUT, exist_ok=True)
    with tempfile.TemporaryDirectory(prefix="bnzref_") as tmp:
        for rel in FILES:
            with open(os.path.join(ref_root, rel)) as f:
                text = f.read()
            dst = os.path.join(tmp, rel)
            os.makedirs(os.path.dirname(dst), exist_ok=True)
            with open(dst, "w") as f:
                f.write(_patch(rel, text))
        for mfield, name in ((1, "libbnzref.so"), (0, "libbnzref_hydro.so")):
            objs = []
            bdir = os.path.join(tmp, "obj_m%d" % mfield)
            os.makedirs(bdir, exist_ok=True)
            for rel in ("src/mhd/eos_c.c", "src/mhd/fluxes_c.c", "src/coordinates/reconstr_c.c"):
                obj = os.path.join(bdir, os.path.basename(rel).replace(".c", ".o"))
                cmd = ["gcc"] + CFLAGS + ["-DMFIELD=%d" % mfield,
                                          "-I" + os.path.join(tmp, "src", "mhd"), "-c",
                                          os.path.join(tmp, rel), "-o", obj]
                subprocess.run(cmd, check=True)
                objs.append(obj)
            lib = os.path.join(OUT, name)
            subprocess.run(["gcc", "-shared", "-Wl,--allow-multiple-definition", "-o", lib]
                           + objs + ["-lm"], check=True)
            if not quiet:
                print("build_ref: built", lib)
    # earlier builds kept their intermediates here: only the libraries stay
    for d in ("src", "obj_m0", "obj_m1"):
        if os.path.isdir(os.path.join(OUT, d)):
            shutil.rmtree(os.path.join(OUT, d))
    return True


if __name__ == "__main__":
    ok = build(sys.argv[1] if len(sys.argv) > 1 else None)
    sys.exit(0 if ok else 1)
