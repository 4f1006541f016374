"""The CLI (beedrill_b200/bin/hybrid_bfs) with the reference's flags and
output lines, plus --batched and --algorithm learned."""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "beedrill_b200", "bin", "hybrid_bfs")


def _run(*args):
    if not os.path.exists(CLI):
        pytest.skip("CLI not built")
    out = subprocess.run([CLI, *args], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                         timeout=300)
    return out.returncode, out.stdout


def _edges(text):
    return [int(x) for x in re.findall(r"Traversed (\d+) edges", text)]


@pytest.mark.parametrize("alg", ["beamer_hybrid", "migrating_threads", "bottom_up", "learned"])
def test_cli_runs_and_checks(alg):
    rc, out = _run("--rmat_scale", "14", "--num_trials", "4", "--algorithm", alg, "--check_results")
    assert rc == 0, out
    assert out.count("PASS") == 4 and "FAIL" not in out
    assert len(_edges(out)) == 4
    assert "Harmonic mean over all trials" in out


def test_cli_batched_matches_one_by_one():
    rc1, one = _run("--rmat_scale", "14", "--num_trials", "70", "--degree_order")
    rc2, bat = _run("--rmat_scale", "14", "--num_trials", "70", "--hub_layout", "--batched",
                    "--algorithm", "learned", "--check_results")
    assert rc1 == 0 and rc2 == 0, (one, bat)
    assert bat.count("PASS") == 70 and "FAIL" not in bat
    assert _edges(one) == _edges(bat)


def test_cli_rejects_a_bad_policy_file(tmp_path):
    bad = tmp_path / "p.json"
    bad.write_text('{"params": [0.5]}')
    rc, out = _run("--rmat_scale", "10", "--algorithm", "learned", "--policy_file", str(bad))
    assert rc != 0 and "policy file" in out
