"""The C++ drop-in classes (include/fm_dropin.hpp) behind the reference's own
set-up and loop (tests/dropin/dropin_main.cpp, a transcription of
src/main.cpp's structure): the header compiles and links against libfm.so on
the CPU; on the GPU the program's fields and outlet CSV equal the Python
binding's run of the same problem (FP64: bit for bit)."""
import os
import subprocess

import numpy as np
import pytest

from fluidmaxxer_b200 import problems, synth, vti

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "dropin", "dropin_main.cpp")
LIBDIR = os.path.join(ROOT, "fluidmaxxer_b200")


def _build(tmp_path):
    exe = str(tmp_path / "dropin_main")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC,
                        "-L", LIBDIR, "-lfm", f"-Wl,-rpath,{LIBDIR}", "-o", exe],
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    assert "warning" not in r.stdout, r.stdout
    return exe


def test_dropin_header_compiles_and_links(tmp_path):
    _build(tmp_path)


def test_reference_interface_subclasses_compile_unchanged(tmp_path):
    """Collision operators and boundaries written against the reference's
    virtual interfaces (initEq / collideStream / apply with its signatures)
    compile and link against the drop-in header."""
    src = os.path.join(ROOT, "tests", "dropin", "reference_interfaces.cpp")
    exe = str(tmp_path / "reference_interfaces")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), src,
                        "-L", LIBDIR, "-lfm", f"-Wl,-rpath,{LIBDIR}", "-o", exe],
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    assert "warning" not in r.stdout, r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_dropin_main_equals_python_binding(tmp_path, prec):
    from fluidmaxxer_b200 import lattice

    nx, ny, nz, steps, every = 40, 16, 12, 300, 50
    solid = synth.bernoulli(nx, ny, nz, 0.3, 5, fluid_lo=4, fluid_hi=4, walls=True)
    vti.write_vti(tmp_path / "geometry.vti", nx, ny, nz, solid.astype(np.float64), name="solid", binary=False)
    exe = _build(tmp_path)
    r = subprocess.run([exe, str(tmp_path), str(steps), str(every)] + (["f32"] if prec == "f32" else []),
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    # the boundaries written against the reference's interface were applied
    # once per phase of every step, with the step index of that step
    assert f"apply ns {steps} {steps} 0 ad {steps} {steps} 0" in r.stdout, r.stdout
    n = nx * ny * nz
    got = np.fromfile(tmp_path / "fields.bin", dtype=np.float64).reshape(6, n)

    p = problems.Problem(nx=nx, ny=ny, nz=nz, solid=solid, tau=0.8, tau_ad=0.7, u_in=(0.01, 0.0, 0.0),
                         isotherm="linear", k_henry=2.0, k_a=0.01, sample_every=every, steps=steps)
    L = lattice.from_problem(p, prec)
    L.step(steps)
    ref = L.fields()
    bt = L.breakthrough()
    L.close()
    for i, k in enumerate(("rho", "ux", "uy", "uz", "phi", "q")):
        assert np.array_equal(got[i], ref[k]), k
    rows = np.loadtxt(tmp_path / "outlet.csv", delimiter=",", skiprows=1)
    assert np.array_equal(rows[:, 0], np.arange(0, steps + 1, every))
    assert np.allclose(rows[:, 1], 0.5 * rows[:, 0])
    assert np.allclose(rows[:, 2], bt, rtol=1e-5, atol=1e-12)     # the CSV prints 6 significant digits
    assert np.all(rows[:, 3] <= rows[:, 2] + 1e-12) and np.all(rows[:, 4] >= rows[:, 2] - 1e-12)
