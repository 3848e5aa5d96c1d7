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
def test_run_writes_density(tmp_path, tpo_built):
    import numpy as np
    src = (REPO / "examples" / "mbb_60x20.yaml").read_text().replace(
        "max_iterations: 100", "max_iterations: 3")
    y = tmp_path / "p.yaml"
    y.write_text(src)
    assert cli.main(["run", str(y), "--output", str(tmp_path / "out"), "--quiet"]) == 0
    rho = np.load(tmp_path / "out" / "density_final.npy")
    assert rho.shape == (1200,) and 0.001 <= rho.min() and rho.max() <= 1.0
