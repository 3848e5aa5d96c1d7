"""CLI: same subcommands and exit codes as the reference's (cli.py:22-144)."""

import pytest

from conftest import REPO
from toptimization_b200 import cli


def test_validate_ok(capsys):
    assert cli.main(["validate", str(REPO / "examples" / "bridge_2048x1024.yaml")]) == 0
    out = capsys.readouterr().out
    assert "is valid" in out and "4,200,450" in out and "2,097,152" in out


def test_validate_missing_and_invalid(tmp_path, capsys):
    assert cli.main(["validate", str(tmp_path / "nope.yaml")]) == 1
    bad = tmp_path / "bad.yaml"
    bad.write_text("domain: {nelx: 4, nely: 2}\nsolver: {preconditioner: ilu}\n")
    assert cli.main(["validate", str(bad)]) == 1
    assert "Validation failed" in capsys.readouterr().err


@pytest.mark.parametrize("backend", ["cpu", "metal", "vulkan"])
def test_run_rejects_non_cuda_backends(backend, capsys):
    rc = cli.main(["run", str(REPO / "examples" / "mbb_60x20.yaml"), "--backend", backend])
    assert rc == 1
    assert "CUDA only" in capsys.readouterr().err


def test_no_command_prints_help(capsys):
    assert cli.main([]) == 0
    assert "run" in capsys.readouterr().out


@pytest.mark.gpu
def test_run_outputs_match_reference(tmp_path, tpo_built):
    """`run` on the MBB 60x20 example writes density_final.npy (the flat
    design density, as the reference's simp.py:294-295 saves it) and
    history.json; both match the reference's own FP64 run of the same file
    (tests/golden/ref_run_mbb_60x20.npz) to the 100-iteration bounds of the
    library-level test (tests/test_gpu_simp.py)."""
    import json

    import numpy as np

    from conftest import golden
    out = tmp_path / "out"
    assert cli.main(["run", str(REPO / "examples" / "mbb_60x20.yaml"), "--output", str(out),
                     "--quiet"]) == 0
    g = golden("ref_run_mbb_60x20")
    rho = np.load(out / "density_final.npy")
    assert rho.shape == (1200,) and rho.dtype == np.float64
    hist = json.loads((out / "history.json").read_text())
    c = np.array(hist["compliance"])
    assert len(c) == len(g["compliance"]) == 100
    assert np.max(np.abs(c - g["compliance"]) / g["compliance"]) < 1e-9
    assert np.abs(np.array(hist["volume"]) - g["volume"]).max() < 1e-9
    assert np.abs(rho - g["rho_final"]).max() < 2.5e-8
