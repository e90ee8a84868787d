"""The JNI glue (artisynth_core_b200/jni/B200FemJNI.cc) compiles against
the C ABI header, and every native method it defines forwards to entry
points that include/b200fem.h declares and libb200fem.so exports.  No JDK is
installed here: the compile uses tests/jni_decl/jni.h, which declares the
JNI types and calls the shim uses (a JDK build uses the real jni.h)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "artisynth_core_b200", "jni", "B200FemJNI.cc")


def test_shim_compiles(tmp_path):
    obj = tmp_path / "B200FemJNI.o"
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-Wextra", "-Werror", "-c",
                        "-I", os.path.join(ROOT, "tests", "jni_decl"), "-I", os.path.join(ROOT, "include"),
                        SHIM, "-o", str(obj)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    syms = subprocess.run(["nm", "-g", "--defined-only", str(obj)], capture_output=True, text=True).stdout
    natives = set(re.findall(r"\b(Java_maspack_solvers_B200Fem(?:Solver|Server)_\w+)", syms))
    assert len(natives) >= 40, sorted(natives)


def test_shim_calls_only_declared_entry_points():
    from artisynth_core_b200 import _lib as L

    src = open(SHIM).read()
    called = set(re.findall(r"\b(b200fem_[a-z0-9_]+)\s*\(", src))
    declared = set(L.header_symbols())
    assert called and called <= declared, sorted(called - declared)
    # the hot-path entry points of the reference-facing binding are all bound
    for name in ("b200fem_create", "b200fem_destroy", "b200fem_last_error", "b200fem_set_mesh",
                 "b200fem_set_material", "b200fem_build", "b200fem_get_crs_indices", "b200fem_get_slot_map",
                 "b200fem_update_stress_stiffness", "b200fem_backward_euler_step",
                 "b200fem_backward_euler_step_host", "b200fem_pcg_solve", "b200fem_spmv"):
        assert name in called, name


@pytest.mark.skipif(not os.environ.get("JAVA_HOME"), reason="no JDK: the real jni.h build needs JAVA_HOME")
def test_shim_builds_with_jdk(tmp_path):
    jh = os.environ["JAVA_HOME"]
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-I", os.path.join(jh, "include"),
                        "-I", os.path.join(jh, "include", "linux"), "-I", os.path.join(ROOT, "include"), SHIM,
                        "-o", str(tmp_path / "libB200FemJNI.so")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
