"""Command-line contract of bin/scout_<problem> and run.sh that needs no GPU."""
import os
import subprocess

import pytest

from conftest import ROOT, SAMPLE

PROBLEMS = ["mis", "coloring", "bfs", "cc"]


@pytest.mark.parametrize("p", PROBLEMS)
def test_usage_with_too_few_arguments(p):
    exe = os.path.join(ROOT, "bin", f"scout_{p}")
    if not os.path.exists(exe):
        pytest.skip("CLIs not built")
    r = subprocess.run([exe, "a", "b"], capture_output=True, text=True)
    assert r.returncode == 1
    assert f"<initial_{p}_context.txt> <batch_folder> <num_batches> <gpu_device_id>" in r.stderr


def test_run_sh_argument_errors():
    sh = os.path.join(ROOT, "run.sh")
    r = subprocess.run(["bash", sh], capture_output=True, text=True)
    assert r.returncode == 1 and "--problem=mis|coloring|bfs|cc is required" in r.stderr
    r = subprocess.run(["bash", sh, "--problem=tsp"], capture_output=True, text=True)
    assert r.returncode == 1 and "must be mis, coloring, bfs, or cc" in r.stderr
    r = subprocess.run(["bash", sh, "--problem=bfs", "--graph=/nonexistent.egr", f"--init={SAMPLE}/sample_bfs.txt",
                        f"--batch={SAMPLE}/batches"], capture_output=True, text=True)
    assert r.returncode == 1 and "graph file not found" in r.stderr
    r = subprocess.run(["bash", sh, "--problem=bfs", "--bogus"], capture_output=True, text=True)
    assert r.returncode == 1 and "unrecognized argument" in r.stderr
    r = subprocess.run(["bash", sh, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--num-batches" in r.stderr
