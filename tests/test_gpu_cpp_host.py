"""GPU: the C++ host mirror (include/tspg_trident.hpp) compiled against the C ABI
and run: the reference's test_compression.cu known answers and sp_mma stages."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_host_mirror(tmp_path):
    exe = str(tmp_path / "test_trident_host")
    lib = os.path.join(ROOT, "trident_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "cpp", "test_trident_host.cpp"), "-o", exe, "-L", lib, "-ltspg",
           "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{lib}"]
    env = dict(os.environ)
    env.pop("CXX", None)
    subprocess.run(cmd, check=True, env=env)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout, r.stderr)
    assert r.returncode == 0 and "ALL OK" in r.stdout
