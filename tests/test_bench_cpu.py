"""Host logic of bench.py that feeds the bench line: the ncu traffic ingest
(unit row of the raw CSV, the INT8 and DMMA operation counters)."""
import csv
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _write(path, head, units, rows):
    with open(path, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(head)
        w.writerow(units)
        for r in rows:
            w.writerow(r)


def test_ingest_scales_by_the_unit_row_and_counts_dmma_as_512_flops(tmp_path):
    src, out = tmp_path / "raw.csv", tmp_path / "traffic.json"
    head = ["ID", "Kernel Name", "dram__bytes_read.sum", "dram__bytes_write.sum",
            "sm__inst_executed_pipe_tensor_subpipe_dmma.sum", "sm__ops_path_tensor_op_utcimma_src_int8_sparsity_off.sum"]
    units = ["", "", "Mbyte", "Kbyte", "inst", ""]
    _write(src, head, units, [
        ["0", "void xg_batch_sched_kernel<32>(CUtensorMap_st, int)", "2.0", "500", "1000", ""],
        ["1", "xg_sliced_left_kernel(CUtensorMap_st)", "1.5", "0", "", "3000000"],
        ["2", "xg_sliced_left_kernel(CUtensorMap_st)", "0.5", "0", "", "1000000"],
    ])
    bench.ingest_ncu(str(src), "case", "cmd", out_path=str(out))
    d = json.load(open(out))
    sch = d["xg_batch_sched_kernel"]
    assert sch["dram_bytes"] == 2.0e6 + 500e3
    assert sch["ops"] == 512.0 * 1000
    assert abs(sch["dram_bytes_per_op"] - 2.5e6 / 512e3) < 1e-12
    sl = d["xg_sliced_left_kernel"]
    assert sl["launches"] == 2 and sl["dram_bytes"] == 2.0e6 and sl["ops"] == 4.0e6
    assert sl["case"] == "case" and sl["command"] == "cmd"
