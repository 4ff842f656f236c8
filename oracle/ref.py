"""Loader for DUCC's own CPU NUFFT and w-gridder, built from the reference
sources by ``oracle/Makefile`` into ``oracle/_ref`` - TEST INFRASTRUCTURE ONLY.

``load()`` returns the compiled module (or None when it was not built).  It
exposes DUCC's ``nufft`` functions and plan class unchanged (``nu2u``, ``u2nu``,
``plan``, ``bestEpsilon``), its ``wgridder`` module (``vis2dirty``,
``dirty2vis``, ``ms2dirty``, ``dirty2ms``) and the read-only probes of
``ref_glue.cc``.
The widest ISA variant that the running CPU supports is picked.
"""
import importlib.util
import os
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
_MOD = None


def _cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def _candidates():
    flags = _cpu_flags()
    v4 = {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags
    v3 = {"avx2", "fma", "bmi2"} <= flags
    out = []
    if v4:
        out.append("ducc_ref_v4")
    if v3:
        out.append("ducc_ref_v3")
    return out


def load():
    """The compiled reference module, or None if it is absent."""
    global _MOD
    if _MOD is not None:
        return _MOD
    if not os.path.isdir(REF_DIR):
        return None
    files = os.listdir(REF_DIR)
    for name in _candidates():
        hit = [f for f in files if f.startswith(name + ".") and f.endswith(".so")]
        if not hit:
            continue
        spec = importlib.util.spec_from_file_location(name, os.path.join(REF_DIR, hit[0]))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules.setdefault(name, mod)
        _MOD = mod
        return mod
    return None


def simd_lanes_double():
    """SIMD lanes the loaded reference build uses for float64 (its parameter
    cost model depends on it: 8 with AVX-512, 4 with AVX2)."""
    mod = load()
    if mod is None:
        return None
    return 8 if mod.__name__.endswith("v4") else 4
