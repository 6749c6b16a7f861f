"""Transmit split of a job into launches of fewer than 2^31 channel samples
(mach_b200/csrc/das_split.h), shared by the allocating entry points and the allocation-free
one.  The header is host C++ only; the test compiles a small driver with g++ and checks the
launch count and each launch's first transmit and transmit count."""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
LIMIT = 2**31 - 1

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include "das_split.h"
int main(int argc, char** argv) {
    const long long per_tx = std::atoll(argv[1]), n_tx = std::atoll(argv[2]);
    const mach_b200::TransmitSplit s = mach_b200::split_transmits(per_tx, n_tx);
    std::printf("%lld %lld\n", static_cast<long long>(s.max_tx), static_cast<long long>(s.n_launch));
    for (long long k = 0; k < s.n_launch; ++k)
        std::printf("%lld %lld\n", static_cast<long long>(mach_b200::launch_first_tx(s, k)),
                    static_cast<long long>(mach_b200::launch_tx_count(s, n_tx, k)));
    return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("split")
    src = d / "split.cc"
    src.write_text(DRIVER)
    exe = d / "split"
    subprocess.run([gxx, "-std=c++17", "-O1", f"-I{REPO / 'mach_b200' / 'csrc'}", str(src), "-o", str(exe)],
                   check=True)
    return exe


def run(exe, per_tx, n_tx):
    out = subprocess.run([str(exe), str(per_tx), str(n_tx)], check=True, capture_output=True, text=True).stdout
    rows = [tuple(int(v) for v in line.split()) for line in out.strip().splitlines()]
    (max_tx, n_launch), launches = rows[0], rows[1:]
    assert len(launches) == n_launch
    return max_tx, n_launch, launches


def expected(per_tx, n_tx):
    max_tx = max(1, LIMIT // max(per_tx, 1))
    n_launch = -(-max(n_tx, 1) // max_tx)
    return max_tx, n_launch


@pytest.mark.parametrize("n_launch", [1, 2, 64, 65])
def test_launch_count_boundaries(driver, n_launch):
    """Jobs that need exactly 1, 2, 64 and 65 launches (the allocation-free call stops at 64)."""
    per_tx = 2**20 * 3  # 3 Mi samples per transmit: 682 transmits per launch
    max_tx = LIMIT // per_tx
    for n_tx in (max_tx * (n_launch - 1) + 1, max_tx * n_launch):
        got_max, got_n, launches = run(driver, per_tx, n_tx)
        assert (got_max, got_n) == (max_tx, n_launch) == expected(per_tx, n_tx)
        # launches tile the transmits in order, each below the sample limit
        assert [f for f, _ in launches] == [k * max_tx for k in range(n_launch)]
        assert sum(c for _, c in launches) == n_tx
        assert all(0 < c <= max_tx and c * per_tx <= LIMIT for _, c in launches)


def test_offsets_of_a_ragged_last_launch(driver):
    per_tx = 128 * 1024 * 200  # one Doppler transmit: 26.2 M samples, 81 per launch
    max_tx, n_launch, launches = run(driver, per_tx, 200)
    assert (max_tx, n_launch) == (81, 3)
    assert launches == [(0, 81), (81, 81), (162, 38)]


def test_degenerate_jobs(driver):
    assert run(driver, 1000, 0)[1:] == (1, [(0, 0)])  # no transmits: one empty launch
    assert run(driver, 0, 5)[:2] == (LIMIT, 1)  # empty transmits
    assert run(driver, LIMIT + 5, 3)[:2] == (1, 3)  # one transmit per launch at least
