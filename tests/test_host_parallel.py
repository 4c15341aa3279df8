"""Host threading of the set-up (tetfit_b200/csrc/host_parallel.hpp): the
worker pool's job hand-off, concurrent callers and the stable parallel sort,
through a small C++ checker (tests/host_parallel_check.cpp) built with the
host compiler.  The set-up's results rely on these being exact: every index
of a loop runs once, and sorts keep the order of equal keys."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    cxx = os.environ.get("CXX") or shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path_factory.mktemp("hp") / "host_parallel_check")
    subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", os.path.join(HERE, "host_parallel_check.cpp"), "-o", exe],
                   check=True)
    return exe


def test_pool_jobs_sort_exact(checker):
    r = subprocess.run([checker, "20000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_pool_under_oversubscription(checker):
    """Several checkers at once on the same cores: late workers and busy
    pools are the cases where a job hand-off can lose or repeat a task."""
    procs = [subprocess.Popen([checker, "8000"], stdout=subprocess.PIPE, text=True) for _ in range(6)]
    for p in procs:
        out, _ = p.communicate(timeout=300)
        assert p.returncode == 0 and out.strip() == "ok", out
