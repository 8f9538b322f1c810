"""The C++ host mirror (host/sphgpu.hpp) compiles against the C ABI and
drives the modules like the reference's Solver."""
import os
import subprocess

import pytest

from conftest import PKG, ROOT

import oracle  # noqa: E402  (conftest puts oracle/ on sys.path)


def _build(tmp_path):
    exe = tmp_path / "host_mirror"
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "host"),
           os.path.join(ROOT, "tests", "cpp", "host_mirror.cpp"), "-L", PKG, "-lsphgpu", f"-Wl,-rpath,{PKG}",
           "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_host_mirror_compiles_and_fails_loudly_without_device(G, tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    if G.device_ok():
        pytest.skip("a device is present (covered by the gpu test)")
    assert r.returncode == 3, r.stdout + r.stderr


@pytest.mark.gpu
def test_host_mirror_runs_steps(gpu, tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "neighbours(0)=" in r.stdout


def test_reference_side_binding_compiles(tmp_path):
    """The reference-side binding (host/gpu_modules.hpp: the four GPU Module
    subclasses and the particle sync) compiles against the reference's own
    headers (include/module.hpp, simulation.hpp, parameters.hpp, particle.hpp,
    exception.hpp) and include/sphgpu.h, with the flags the reference's
    sources build with."""
    refdir = oracle.refdir()
    if not os.path.isdir(os.path.join(refdir, "include")):
        pytest.skip("the reference's headers are not mounted here")
    src = tmp_path / "use_gpu_modules.cpp"
    src.write_text('#include "gpu_modules.hpp"\n'
                   "int main() { sph::SPHParameters p{}; (void)sph::GpuContext::params(p); return 0; }\n")
    r = subprocess.run(["g++", "-std=c++14", "-fsyntax-only", "-fopenmp", "-DDIM=3", "-include", "string",
                        "-include", "limits", "-I", os.path.join(refdir, "include"), "-I",
                        os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "host"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
