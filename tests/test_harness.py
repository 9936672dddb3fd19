"""The standalone C harness (faceted-hypersara_b200/harness/fhs_harness.c):
a plain C99 program over the C ABI, configured by a JSON file in the layout
of the reference's imaging/default_parameters.json plus a "harness" section.

CPU: configuration parsing (--dry-run touches no GPU) and error exits.
GPU: small FHS / HS / SARA problems, preconditioned and visibility-gridding
variants, solved to the reference's stopping rule; the reconstruction SNR
against the synthetic ground truth stands in for correctness (the solver
arithmetic itself is checked against the oracle by the other GPU tests).
"""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "faceted-hypersara_b200", "fhs_b200", "fhs_harness")
CONFIG = os.path.join(ROOT, "faceted-hypersara_b200", "harness", "example_config.json")

needs_harness = pytest.mark.skipif(not os.path.exists(HARNESS), reason="harness not built (run build())")


def _run(*args, timeout=600):
    r = subprocess.run([HARNESS, *args], capture_output=True, text=True, timeout=timeout)
    return r.returncode, r.stdout, r.stderr


@needs_harness
def test_dry_run_reads_the_reference_layout():
    rc, out, err = _run(CONFIG, "--dry-run")
    assert rc == 0, err
    d = json.loads(out)
    assert d["algo"] == "fhs" and (d["Ny"], d["Nx"], d["L"]) == (128, 128, 8)
    assert (d["oy"], d["J"], d["nlevel"]) == (2, 7, 4)
    assert d["pdfb_max_iter"] == 150 and d["reweighting_max_iter"] == 1 and d["elipse_proj_max_iter"] == 20
    rc, out, err = _run(CONFIG, "algo=sara", "Ny=64", "dr=1", "--dry-run")
    d = json.loads(out)
    assert rc == 0 and d["algo"] == "sara" and d["L"] == 1 and d["Qy"] == 1 and d["Ny"] == 64 and d["dr"] == 1


@needs_harness
def test_configuration_errors_exit_1(tmp_path):
    bad = tmp_path / "bad.json"
    bad.write_text('[{"pdfb": {"max_iter": }]')
    assert _run(str(bad), "--dry-run")[0] == 1
    assert _run(str(tmp_path / "missing.json"), "--dry-run")[0] == 1
    assert _run(CONFIG, "n_blocks=17", "--dry-run")[0] == 1
    assert _run(CONFIG, "precond=1", "dr=1", "--dry-run")[0] == 1
    assert _run(CONFIG, "vis_fraction=1e-9")[0] == 1   # rejected before any GPU call


@pytest.mark.gpu
@needs_harness
@pytest.mark.parametrize("args,min_snr", [
    (("Ny=64", "Nx=64", "L=4"), 18.0),
    (("algo=hs", "Ny=64", "Nx=64", "L=4"), 18.0),
    (("algo=sara", "Ny=64", "Nx=64"), 20.0),
    (("Ny=64", "Nx=64", "L=4", "precond=1"), 18.0),
    (("Ny=64", "Nx=64", "L=4", "dr=1", "vis_fraction=2"), 18.0),
])
def test_harness_solves(tmp_path, args, min_snr):
    out = tmp_path / "x.bin"
    rc, so, err = _run(CONFIG, *args, f"output={out}")
    assert rc == 0, err
    d = json.loads(so.strip().splitlines()[-1])
    assert d["n_iter"] >= 1 and d["snr_db"] > min_snr, d
    assert out.stat().st_size == 8 * d["Ny"] * d["Nx"] * d["L"]


def test_mex_gateway_compiles_against_the_abi():
    """faceted-hypersara_b200/mex/fhs_mex.c type-checks against include/fhs_b200.h
    (MATLAB's mex.h is absent here: tests/mex_stub/mex.h declares the calls it uses)."""
    import shutil
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    r = subprocess.run([cc, "-fsyntax-only", "-std=c99", "-Wall", "-Wextra", "-Werror",
                        "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "tests", "mex_stub"),
                        os.path.join(ROOT, "faceted-hypersara_b200", "mex", "fhs_mex.c")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@needs_harness
def test_dry_run_accepts_a_single_object(tmp_path):
    """A configuration may also be one JSON object holding the sections."""
    cfg = tmp_path / "one.json"
    cfg.write_text(json.dumps({"pdfb": {"max_iter": 77}, "sara": {"nlevel": 3},
                               "aux_global": {"measop_flag_visibility_gridding": True},
                               "harness": {"algo": "hs", "Ny": 96, "Nx": 80, "L": 5, "snr_db": 30}}))
    rc, out, err = _run(str(cfg), "--dry-run")
    assert rc == 0, err
    d = json.loads(out)
    assert (d["algo"], d["Ny"], d["Nx"], d["L"], d["Qy"]) == ("hs", 96, 80, 5, 1)
    assert d["pdfb_max_iter"] == 77 and d["nlevel"] == 3 and d["dr"] == 1 and d["snr_db"] == 30


def test_matlab_wrappers_match_the_gateway_and_the_reference_signatures():
    """Every fhs_mex command the .m wrappers call exists in the gateway, and
    each wrapper keeps the argument list of the reference function it stands
    in for (src/*.m, lib/operators/*.m)."""
    import re
    mex_dir = os.path.join(ROOT, "faceted-hypersara_b200", "mex")
    gateway = open(os.path.join(mex_dir, "fhs_mex.c")).read()
    commands = set(re.findall(r'!strcmp\(cmd, "(\w+)"\)', gateway))
    expected = {
        "apply_direct_operator": "Fx, G, Lambda",
        "apply_adjoint_operator": "y, G, Lambda",
        "HS_forward_operator_G": "x, G, W, A, flag_visibility_gridding, Lambda",
        "HS_adjoint_operator_G": "y, G, W, At, N, M, flag_visibility_gridding, Lambda",
        "proj_l2ball": "x, eps, y",
        "nuclear_norm": "x",
        "compute_sara_prior": "x, Psit, n_wavelet_coefficients",
        "update_dual_data_fidelity": "v2, y, x, Fx_old, proj, A, At, G, W, pU, epsilon, elipse_proj_max_iter, "
                                     "elipse_proj_min_iter, elipse_proj_eps, sigma22, "
                                     "flag_dimensionality_reduction, Lambda",
        "facetHyperSARA": "y, epsilon, A, At, pU, G, W, param, Qx, Qy, K, wavelet, filter_length, nlevel, "
                          "window_type, spectral_chunk, n_channels, overlap_size, M, N, oy, ox, warmstart_name, "
                          "checkpoint_name, flag_dimensionality_reduction, Lambda, varargin",
        "hyperSARA": "y, epsilon, A, At, pU, G, W, param, K, wavelet, nlevel, spectral_chunk, n_channels, M, N, "
                     "oy, ox, warmstart_name, checkpoint_name, flag_dimensionality_reduction, Sigma, varargin",
        "sara": "y, epsilon, A, At, pU, G, W, Psi, Psit, param, warmstart_name, checkpoint_name, alph, "
                "flag_dimensionality_reduction, Lambda, varargin",
    }
    mdir = os.path.join(mex_dir, "matlab")
    used = set()
    for f in sorted(os.listdir(mdir)):
        src = open(os.path.join(mdir, f)).read()
        used |= set(re.findall(r"fhs_mex\('(\w+)'", src))
        name = f[:-2]
        if name in expected:
            head = src[:src.index(")")].replace("...", " ")
            args = re.sub(r"\s+", " ", head[head.index(name + "(") + len(name) + 1:]).strip()
            assert args == expected[name], (name, args)
    assert used and used <= commands, used - commands
    assert set(expected) <= {f[:-2] for f in os.listdir(mdir)}
