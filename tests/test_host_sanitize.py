"""The library's host code under AddressSanitizer and UndefinedBehaviorSanitizer, on the CPU.

libqas.so is rebuilt from the same sources with -fsanitize=address,undefined on the host side
(device code as PTX only: nothing here launches a kernel), and tests/native/host_plans.cpp
drives its host-only entry points -- qas_step_host's wave plans for 21..700 planes and 0..64
windows in both lane modes, the ghost-fill maps of every group, field and axis and the slab
plans of 1-4 parts for 3000 random grids and boundary-flag mixes, the status strings -- with
leak detection on and any report fatal."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_host_code_clean_under_asan_ubsan(tmp_path):
    from qasmhd_b200.build import nvcc
    try:
        nv = nvcc()
    except FileNotFoundError:
        pytest.skip("nvcc not available")
    lib = str(tmp_path / "libqas_san.so")
    subprocess.run([nv, "-gencode", "arch=compute_100a,code=compute_100a", "-O1", "-g", "--fmad=false",
                    "-std=c++17", "-Xcompiler", "-fPIC,-fsanitize=address,-fsanitize=undefined,-fno-omit-frame-pointer",
                    "-shared", "-cudart=static", "-o", lib, os.path.join(ROOT, "qasmhd_b200", "csrc", "qas_api.cu"),
                    "-Xlinker", "-fsanitize=address,-fsanitize=undefined"],
                   check=True, cwd=str(tmp_path), timeout=900)
    exe = str(tmp_path / "host_plans")
    subprocess.run(["g++", "-O1", "-g", "-std=c++17", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "native", "host_plans.cpp"),
                    "-L", str(tmp_path), "-lqas_san", f"-Wl,-rpath,{tmp_path}", "-o", exe], check=True, timeout=300)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:halt_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    r = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "host plans ok" in r.stdout
    assert "runtime error" not in r.stderr and "ERROR: AddressSanitizer" not in r.stderr
