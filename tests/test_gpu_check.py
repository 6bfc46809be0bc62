"""Index-checking build (libsfac_check.so, -DSPME_CHECK): every kernel path
runs with its grid, bucket, atom and table indices tested, and no check may
fail.  A failed check records its site and index in an error word and skips
the access (no trap), so this test faults no GPU even if a check fires.  The
library runs in a child process (tests/check_cases.py) so it never shares a
process with the product libsfac.so."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def check_run(oracle_built):
    from ewaldcorrel_b200 import build

    if not os.path.exists(build.LIB_CHECK):
        build.build(check=True)
    env = dict(os.environ, EWALDCORREL_LIBSFAC=build.LIB_CHECK)
    r = subprocess.run([sys.executable, os.path.join(HERE, "check_cases.py")], env=env, capture_output=True,
                       text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_the_checking_build_checks(check_run):
    assert check_run["library"].endswith("libsfac_check.so")
    assert check_run["enabled"] == 1
    assert check_run["selftest"] == 0  # a planted failure comes back as (site, index)
    assert check_run["start"][0] == 0


def test_no_index_check_fails_on_any_path(check_run):
    bad = [c for c in check_run["cases"] if c["module"] != 0]
    assert not bad, bad
    assert len(check_run["cases"]) == 11


def test_the_checking_build_keeps_parity(check_run):
    for c in check_run["cases"]:
        assert c["energy_rel"] <= 1e-6, c
        assert c["force_rrms"] <= 1e-5, c
        assert c["pot_rrms"] <= 1e-5, c
