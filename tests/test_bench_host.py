"""Host-side legs of bench.py that need no device: the reader leg and the
reference-arm helpers' option mapping."""
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def test_reader_leg_reads_every_sample_file():
    import bench
    wl, q, r = bench.make_workload(2, 300, 2)
    out = bench.reader_run(wl, types.SimpleNamespace(reader_files=120), r)
    assert out["files"] == 120 and out["all_structures_read"]
    assert out["value"] > 0 and out["residues_per_s"] > 0 and out["unit"] == "files/s"


def test_option_mapping_of_the_reference_arms():
    import bench
    a13, a9 = types.SimpleNamespace(speed=13), types.SimpleNamespace(speed=9)
    assert bench.cli_options(a13) == ["--no-detailed-search"]
    assert bench.cli_options(a9) == ["--speed=9"]
    assert bench.lib_options(a13, 5).polish_steps == 5
    assert bench.lib_options(a9, 0)._c().nodetailedsearch == 0
    assert "--no-detailed-search" in bench.options_text(a13)
