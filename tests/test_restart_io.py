"""The reference's restart and output formats (readfiles.cpp:1230-1651):
files the reference program wrote (tests/golden/io, made by
tests/golden/make_io_golden.py: a 2-step MD run of the 4-atom Al cell) are
read and written back byte for byte, and their contents agree with each
other and with the system."""
from __future__ import annotations

from pathlib import Path

import numpy as np

IO = Path(__file__).resolve().parent / "golden" / "io"


def test_restart_round_trip(tmp_path):
    from sqdft_b200.restart_io import read_restart, write_restart

    nproc, rho = read_restart(IO / "tiny.restart")
    assert nproc == 1 and rho.shape == (8 ** 3,)
    # the last SCF iteration's density (PrintSCF runs inside the SCF loop,
    # scf.cpp:162-163) holds the 12 valence electrons of 4 Al to the SCF
    # tolerance (h = 7.78 / 8)
    assert abs(rho.sum() * (7.78 / 8) ** 3 - 12.0) < 1e-5
    write_restart(tmp_path / "x.restart", rho, nproc)
    assert (tmp_path / "x.restart").read_bytes() == (IO / "tiny.restart").read_bytes()


def test_rank_order_of_blocks():
    from sqdft_b200.restart_io import rank_order

    whole = np.arange(2 * 3 * 4, dtype=np.float64).reshape(2, 3, 4)
    # two ranks, z-slabs: rank 0's block first, each z-major
    assert np.array_equal(rank_order([whole[:1], whole[1:]]), whole.reshape(-1))


def test_aout_round_trip(tmp_path):
    from sqdft_b200.restart_io import read_aout, write_aout

    out = read_aout(IO / "tiny.aout")
    assert out.n_atm == 4 and len(out.types) == 1 and out.types[0].symb == "Al" and out.types[0].Z == 3
    write_aout(tmp_path / "x.aout", out)
    assert (tmp_path / "x.aout").read_bytes() == (IO / "tiny.aout").read_bytes()


def test_restart_md_round_trip_and_agrees_with_aout(tmp_path):
    from sqdft_b200.restart_io import read_aout, read_restart_md, write_restart_md

    md = read_restart_md(IO / "tiny.restartMD")
    assert md.step == 2 and md.velocities.shape == (4, 3) and md.stats.shape == (4, 2)
    write_restart_md(tmp_path / "x.restartMD", md)
    assert (tmp_path / "x.restartMD").read_bytes() == (IO / "tiny.restartMD").read_bytes()
    # the same final forces and positions, printed to 14 and 16 digits in .aout
    out = read_aout(IO / "tiny.aout")
    assert np.abs(md.forces - out.forces).max() <= 1e-14
    assert np.abs(md.positions - out.types[0].positions).max() <= 1e-14
