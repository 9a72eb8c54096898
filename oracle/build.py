"""Build the CPU oracle (TEST INFRASTRUCTURE ONLY).

  oracle/liboracle.so          the plain-C restatement (always built)
  oracle/_ref/libnufht_ref.so  the reference's own src/fast_hankel_nufht.c and src/bounds.c,
                               compiled unchanged from the reference tree, linked with the
                               oracle's evaluators (built only where the reference tree exists)

The reference tree is read from $NUFHT_REFERENCE_DIR (default /root/reference).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libnufht_ref.so")
REF_DIR = os.environ.get("NUFHT_REFERENCE_DIR", "/root/reference")
CFLAGS = ["-O2", "-fPIC", "-shared", "-fopenmp", "-std=gnu11"]


def _stale(target, deps):
    return not os.path.exists(target) or os.path.getmtime(target) < max(os.path.getmtime(d) for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("%s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))


def build():
    src = [os.path.join(HERE, "nufht_oracle.c")]
    deps = src + [os.path.join(HERE, "nufht_oracle.h")]
    if _stale(LIB, deps):
        _run(["gcc"] + CFLAGS + src + ["-o", LIB, "-lm"])
    ref_src = [os.path.join(REF_DIR, "src", "fast_hankel_nufht.c"), os.path.join(REF_DIR, "src", "bounds.c")]
    if all(os.path.exists(p) for p in ref_src):
        os.makedirs(os.path.dirname(REF_LIB), exist_ok=True)
        glue = [os.path.join(HERE, "ref_glue.c"), os.path.join(HERE, "nufht_oracle.c")]
        if _stale(REF_LIB, ref_src + glue + [os.path.join(HERE, "nufht_oracle.h")]):
            _run(["gcc"] + CFLAGS + ["-I", os.path.join(REF_DIR, "src"), "-I", HERE] + ref_src + glue
                 + ["-o", REF_LIB, "-lm"])
    return LIB


if __name__ == "__main__":
    build()
    print(LIB, os.path.exists(REF_LIB))
