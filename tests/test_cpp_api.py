"""The C++ integrator API (include/pylith_b200/feassemble.hh) compiles against the C ABI and,
on a GPU, registers kernels by the pylith::fekernels addresses and computes through them."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "integrator_cpp.cc")
CUDA = "/usr/local/cuda"


def build(tmp_path):
    exe = str(tmp_path / "integrator_cpp")
    libdir = os.path.join(ROOT, "pylith_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-o", exe, SRC, f"-I{ROOT}/include", f"-I{CUDA}/include",
           f"-L{libdir}", "-lpylith_b200", f"-Wl,-rpath,{libdir}", f"-L{CUDA}/lib64", "-lcudart"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_api_compiles(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_cpp_api_runs_on_gpu(tmp_path):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    out = subprocess.run([build(tmp_path)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "ok" in out.stdout


def test_reference_compiled_kernels_register_through_the_c_abi(tmp_path):
    """A program compiled against the reference's own libsrc/pylith/fekernels/*.hh (with the
    oracle's four shim headers for PETSc, MPI, pythia and portinfo) registers the addresses of
    the reference's kernels -- the pointers a PyLith material hands to PetscWeakForm -- through
    pl_fekernel_register; a function that computes something else is refused. Host only."""
    src = os.environ.get("PYLITH_SRC")
    if not src or not os.path.isdir(os.path.join(src, "libsrc")):
        pytest.skip("PYLITH_SRC (the PyLith source tree) is not set")
    exe = str(tmp_path / "register_reference")
    libdir = os.path.join(ROOT, "pylith_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-o", exe, os.path.join(ROOT, "tests", "cpp", "register_reference.cc"),
           os.path.join(src, "libsrc", "pylith", "fekernels", "Tensor.cc"),
           f"-I{os.path.join(ROOT, 'oracle', 'ref_shim')}", f"-I{os.path.join(src, 'libsrc')}", f"-I{ROOT}/include",
           f"-L{libdir}", "-lpylith_b200", f"-Wl,-rpath,{libdir}", f"-L{CUDA}/lib64", "-lcudart"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "ok: 15 reference kernels registered" in out.stdout
