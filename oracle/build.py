"""Build the CPU oracle and the boundary checks (TEST INFRASTRUCTURE ONLY).

  oracle/liboracle.so          the plain-C restatement (always built)
  oracle/_ref/libnufht_ref.so  the reference's own src/fast_hankel_nufht.c and src/bounds.c,
                               compiled unchanged from the reference tree, linked with the
                               oracle's evaluators
  oracle/_ref/abi_layout_ref.h sizes and field offsets of the reference header's structs
                               (printed by oracle/abi_layout.c built against that header)
  oracle/_ref/abi_layout_check compiles only when include/nufht_b200.h has the same layouts
  oracle/_ref/test_nufht_ref   the reference's own src/test_nufht.c, compiled unchanged
                               against the reference header and linked with
                               nufht_b200/libnufht_b200.so (the drop-in, proven in C)

Everything under oracle/_ref is built only when $NUFHT_REFERENCE_DIR names the reference
tree; without it only liboracle.so is built (the prebuilt oracle/_ref files are used as
they are).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(REF_OUT, "libnufht_ref.so")
LAYOUT_H = os.path.join(REF_OUT, "abi_layout_ref.h")
LAYOUT_EMIT = os.path.join(REF_OUT, "abi_layout_emit")
LAYOUT_CHECK = os.path.join(REF_OUT, "abi_layout_check")
REF_TEST = os.path.join(REF_OUT, "test_nufht_ref")
PRODUCT_LIB_DIR = os.path.join(ROOT, "nufht_b200")
CFLAGS = ["-O2", "-fPIC", "-shared", "-fopenmp", "-std=gnu11"]


def _stale(target, deps):
    return not os.path.exists(target) or os.path.getmtime(target) < max(os.path.getmtime(d) for d in deps)


def _run(cmd, **kw):
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    if r.returncode != 0:
        raise RuntimeError("%s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout


def reference_dir():
    """The reference tree named by $NUFHT_REFERENCE_DIR, or None."""
    d = os.environ.get("NUFHT_REFERENCE_DIR")
    return d if d and os.path.isdir(os.path.join(d, "src")) else None


def _build_boundary_checks(ref_src_dir):
    hdr = os.path.join(ref_src_dir, "fast_hankel_nufht.h")
    ours = os.path.join(ROOT, "include", "nufht_b200.h")
    src = os.path.join(HERE, "abi_layout.c")
    if _stale(LAYOUT_H, [hdr, src]):
        _run(["gcc", "-std=c11", "-DLAYOUT_EMIT", "-I", ref_src_dir, src, "-o", LAYOUT_EMIT])
        text = _run([LAYOUT_EMIT])
        with open(LAYOUT_H, "w") as f:
            f.write("/* Generated by oracle/build.py from the reference header. */\n" + text)
    if _stale(LAYOUT_CHECK, [LAYOUT_H, ours, src]):
        _run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-I", REF_OUT, src, "-o", LAYOUT_CHECK])
    test_src = os.path.join(ref_src_dir, "test_nufht.c")
    product = os.path.join(PRODUCT_LIB_DIR, "libnufht_b200.so")
    if os.path.exists(test_src) and os.path.exists(product) and _stale(REF_TEST, [test_src, hdr, product]):
        _run(["gcc", "-O2", "-std=gnu11", "-I", ref_src_dir, test_src, "-o", REF_TEST,
              "-L", PRODUCT_LIB_DIR, "-lnufht_b200", "-Wl,-rpath,$ORIGIN/../../nufht_b200", "-lm"])


def build():
    src = [os.path.join(HERE, "nufht_oracle.c")]
    deps = src + [os.path.join(HERE, "nufht_oracle.h")]
    if _stale(LIB, deps):
        _run(["gcc"] + CFLAGS + src + ["-o", LIB, "-lm"])
    ref = reference_dir()
    if ref is None:
        return LIB
    ref_src_dir = os.path.join(ref, "src")
    ref_src = [os.path.join(ref_src_dir, "fast_hankel_nufht.c"), os.path.join(ref_src_dir, "bounds.c")]
    if all(os.path.exists(p) for p in ref_src):
        os.makedirs(REF_OUT, exist_ok=True)
        glue = [os.path.join(HERE, "ref_glue.c"), os.path.join(HERE, "nufht_oracle.c")]
        if _stale(REF_LIB, ref_src + glue + [os.path.join(HERE, "nufht_oracle.h")]):
            _run(["gcc"] + CFLAGS + ["-I", ref_src_dir, "-I", HERE] + ref_src + glue + ["-o", REF_LIB, "-lm"])
        _build_boundary_checks(ref_src_dir)
    return LIB


if __name__ == "__main__":
    build()
    print(LIB, os.path.exists(REF_LIB))
