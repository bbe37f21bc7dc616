"""Results files of the validation campaign (validation/Campaign.hpp:133-139)
written by m3lb_b200.campaign, against a file the reference's own program
wrote: validation/tgv3d_bench.cpp built on the host (tests/golden/dat/, made
by tests/golden/make_validation_golden.py) for D = 32, Re = 1600, u0 = 0.05,
tmax = 1.0 (101 steps, 51 probes), central moments, FP64."""
import math
from pathlib import Path

import pytest

from m3lb_b200 import campaign

GOLD = Path(__file__).resolve().parent / "golden" / "dat" / "tgvb_re1600_d3q27_cm_d32.dat"


def test_writer_formats_numbers_as_printf():
    """Re-printing the fixture's own values with the writer's formats gives
    the fixture's bytes: the header, '%.6f %.8e %.8e %.8e' rows, and the
    first row's undefined dissipation as glibc prints the x86-64 NaN of
    0.0 / 0.0 ('-nan')."""
    lines = GOLD.read_text().splitlines(keepends=True)
    head = campaign.c_format("# t*  Ek*  eps_E  eps_zeta   D=%d Re=%.0f u0=%.4f tau=%.6f\n",
                             32, 1600.0, 0.05, 3 * (0.05 * (32 / (2 * math.pi)) / 1600) + 0.5)
    assert head == lines[0]
    for ln in lines[1:]:
        vals = [float(v) for v in ln.split()]
        assert campaign.c_format("%.6f %.8e %.8e %.8e\n", *vals) == ln
    assert lines[1].split()[2] == "-nan"


def test_open_out_needs_the_results_folder(tmp_path, capsys):
    """open_out opens results/<dir>/<test>_<lat>_<op>.dat when the folder
    exists (and says so) and returns None otherwise, as the reference's fopen
    does."""
    assert campaign.open_out("E_x", "t", "d3q27", "cm", root=str(tmp_path)) is None
    (tmp_path / "results" / "E_x").mkdir(parents=True)
    f = campaign.open_out("E_x", "t", "d3q27", "cm", root=str(tmp_path))
    assert f is not None
    f.close()
    assert (tmp_path / "results" / "E_x" / "t_d3q27_cm.dat").exists()
    assert "-> results/E_x/t_d3q27_cm.dat" in capsys.readouterr().out


@pytest.mark.gpu
def test_tgv_bench_results_file_matches_reference_byte_for_byte(cuda_device, tmp_path):
    """The benchmark run through this library on the device (FP64 populations;
    energy and enstrophy from m3lb_diagnostics) writes the same results file,
    byte for byte, as the reference's program on the host."""
    (tmp_path / "results" / "E_tgv3d_bench").mkdir(parents=True)
    rows = campaign.tgv3d_bench(D=32, Re=1600.0, tmax=1.0, u0=0.05, lat="d3q27", op="cm",
                                storage="f64", root=str(tmp_path))
    assert len(rows) == 51
    got = (tmp_path / "results" / "E_tgv3d_bench" / "tgvb_re1600_d3q27_cm.dat").read_bytes()
    assert got == GOLD.read_bytes()
