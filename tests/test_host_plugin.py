"""The C++ model plugin (LyotropicGPU / NematicGPU) and its standalone build,
without a GPU: the plugin compiles against the reference's own headers (the
drop-in check), the standalone stand-ins reproduce the reference's random
stream and JSON text, massPy reads the files, and the driver fails cleanly
when no device is present."""
import json
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "mass_hd_b200", "host")
COMPAT = os.path.join(HOST, "compat")
NATIVE = os.path.join(ROOT, "tests", "native")
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF = O.REF_DIR
DRIVER = os.path.join(HOST, "_build", "mass-gpu")

LYO_FIELDS = ["ff", "QQxx", "QQyx", "phi", "sigmaXX", "sigmaXY", "sigmaYX", "sigmaYY",
              "sigma_bulk", "sigma_elastic_xx", "sigma_elastic_yx", "sigma_phase_field_xx",
              "sigma_phase_field_yx", "sigma_active_xx", "sigma_active_yx"]


def gxx():
    return shutil.which("g++") or "/usr/bin/g++"


def compile_native(tmp_path, src, extra=()):
    exe = os.path.join(str(tmp_path), os.path.basename(src).replace(".cpp", ""))
    subprocess.run([gxx(), "-std=c++17", "-O1", "-pthread", "-I", COMPAT, os.path.join(NATIVE, src),
                    *extra, "-o", exe], check=True)
    return exe


def test_standalone_driver_builds():
    subprocess.run(["make", "-s", "-C", HOST], check=True)
    assert os.path.exists(DRIVER)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")), reason="reference tree absent")
def test_plugin_compiles_against_reference_headers():
    subprocess.run(["make", "-s", "-C", HOST, "refcheck"], check=True)


def test_bulk_number_format_equals_stringstream(tmp_path):
    """Frame arrays are formatted in parallel chunks by a %.6g conversion of
    our own (std::to_chars near rounding ties); every value must print
    exactly as the reference's `stringstream << v`."""
    exe = compile_native(tmp_path, "format_check.cpp")
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    assert out.split()[-1] == "0", out


@pytest.mark.parametrize("clones", [True, False])
def test_compat_generator_equals_std_mt19937(tmp_path, clones):
    """The standalone build's own Mersenne Twister (block-wise, vectorised)
    and its bulk random_reals give exactly the standard library's
    std::mt19937 / uniform_real_distribution / normal_distribution values,
    in the build whose loader picks the AVX2 block loops where the CPU has
    them and in the baseline-only build."""
    extra = [os.path.join(COMPAT, "random.cpp")] + ([] if clones else ["-DMASS_GPU_NO_CLONES"])
    exe = compile_native(tmp_path, "random_check.cpp", extra)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    assert out.split()[0] == "0", out


def test_compat_random_matches_reference_stream(tmp_path):
    exe = compile_native(tmp_path, "print_random.cpp", [os.path.join(COMPAT, "random.cpp")])
    out = subprocess.run([exe, "42", "64"], check=True, capture_output=True, text=True).stdout
    got = np.array([float(x) for x in out.split()])
    want = np.load(os.path.join(GOLDEN, "configure.npz"))["random_reals_seed42"]
    assert np.array_equal(got, want)


@pytest.mark.parametrize("tag", ["lyo", "nem"])
def test_json_writer_matches_reference_text(tmp_path, tag):
    exe = compile_native(tmp_path, "write_frame.cpp")
    z = np.load(os.path.join(GOLDEN, f"{tag}_frame3_state.npz"))
    d = tmp_path / "fields"
    d.mkdir()
    for k in z.files:
        np.ascontiguousarray(z[k], dtype="<f8").tofile(str(d / f"{k}.bin"))
    out = tmp_path / "frame.json"
    subprocess.run([exe, tag, str(d), str(out)], check=True)
    want = open(os.path.join(GOLDEN, f"{tag}_frame3.json")).read()
    assert out.read_text() == want


def _load_massPy_archive():
    path = os.path.join(REF, "POST", "massPy", "archive.py")
    if not os.path.exists(path):
        pytest.skip("reference massPy absent")
    import importlib.util
    spec = importlib.util.spec_from_file_location("massPy_archive_ref", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_massPy_reads_plugin_json(tmp_path):
    archive = _load_massPy_archive()
    exe = compile_native(tmp_path, "write_frame.cpp")
    z = np.load(os.path.join(GOLDEN, "lyo_frame3_state.npz"))
    d = tmp_path / "fields"
    d.mkdir()
    for k in z.files:
        np.ascontiguousarray(z[k], dtype="<f8").tofile(str(d / f"{k}.bin"))
    run = tmp_path / "run"
    run.mkdir()
    shutil.copy(os.path.join(GOLDEN, "lyo_parameters.json"), str(run / "parameters.json"))
    subprocess.run([exe, "lyo", str(d), str(run / "frame0.json")], check=True)
    ar = archive.loadarchive(str(run))
    fr = ar._read_frame(0)
    assert np.allclose(np.asarray(fr.QQxx), z["QQxx"], rtol=1e-5, atol=1e-6)
    assert np.asarray(fr.ff).shape == (12, 9)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="a GPU is present")
def test_driver_without_device_fails_cleanly(tmp_path):
    subprocess.run(["make", "-s", "-C", HOST], check=True)
    card = tmp_path / "run.dat"
    card.write_text("model = lyotropic\nLX = 8\nLY = 8\nnsteps = 1\nninfo = 1\n"
                    "config = circle\nradius = 2\nconc = 1\nprecision = fp64\n")
    r = subprocess.run([DRIVER, str(card), "-o", str(tmp_path / "out")],
                       capture_output=True, text=True)
    assert r.returncode == 1
    assert "no CUDA device" in r.stderr


def test_driver_rejects_unknown_option_and_model(tmp_path):
    subprocess.run(["make", "-s", "-C", HOST], check=True)
    card = tmp_path / "run.dat"
    card.write_text("model = lyotropic\nLX = 8\nLY = 8\nnsteps = 1\nbogus = 3\n")
    r = subprocess.run([DRIVER, str(card)], capture_output=True, text=True)
    assert r.returncode == 1 and "unknown option 'bogus'" in r.stderr
    card.write_text("model = polar\nLX = 8\nLY = 8\n")
    r = subprocess.run([DRIVER, str(card)], capture_output=True, text=True)
    assert r.returncode == 1 and "can not be found" in r.stderr
