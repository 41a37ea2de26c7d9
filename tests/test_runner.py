"""The benchmark-list runner (cucosma_b200.runner): reading lists in the
reference's TESTS_TO_RUN schema, writing config / nvprof-layout files that the
reference's ResultReader scripts index, and (GPU) running a list with checks."""
import os

import pytest

from cucosma_b200 import runner

HEADER = ",".join(runner.FIELDS)
ROWS = [  # own small configurations in the schema (tile columns as the reference would write them)
    "2,float,float2,float4,96,80,40,128,128,40,8,32,64,8,8,1,1,0,1,4,0,false",
    "2,float,float2,float4,64,64,3000,128,128,750,8,32,64,8,8,4,1,0,1,4,0,true",
    "2,double,double2,double4,50,70,30,128,128,30,8,32,64,8,8,1,1.5,0.5,2,4,0,false",
    "2,float,float2,float4,4,8,5000,4,8,500,8,4,8,1,1,10,1,0,1,4,0,true",
]


def write_list(tmp_path, first="OCCUPANCY"):
    p = tmp_path / "mini.csv"
    p.write_text(HEADER.replace("OCCUPANCY", first) + "\n" + "\n".join(ROWS) + "\n\n")
    return str(p)


@pytest.mark.parametrize("first", ["OCCUPANCY", "ADDITIONAL_OCCUPANCY_SM"])
def test_read_list(tmp_path, first):
    rows = runner.read_list(write_list(tmp_path, first))
    assert len(rows) == 4
    assert rows[1]["M"] == "64" and rows[1]["K"] == "3000" and rows[1]["SPLIT_K"] == "4"
    assert rows[2]["TYPE"] == "double" and rows[2]["BETA"] == "0.5"


def test_config_text_lines_where_the_readers_look(tmp_path):
    import pandas as pd

    row = runner.read_list(write_list(tmp_path))[0]
    p = tmp_path / "config_1.csv"
    p.write_text(runner.config_text(row, "today"))
    df = pd.read_csv(p)
    # the reference's readers take M, N, K, tile sizes from these rows (squaresReader2.py)
    assert df.iloc[10, 0] == "#define M 96" and df.iloc[11, 0] == "#define N 80" and df.iloc[12, 0] == "#define K 40"
    assert df.iloc[13, 0] == "#define THREADBLOCK_TILE_M 128"


def test_nvprof_layout(tmp_path):
    import pandas as pd

    p = tmp_path / "nvprof_1.csv"
    p.write_text(runner.nvprof_text("B200", [(0.0, 10.5, "cublas[torch.matmul]"), (0.0, 7.25, "cosmaSgemm[x]")]))
    df = pd.read_csv(p, skiprows=3)
    assert df["Name"][1] == "cublas[torch.matmul]"  # row 0 is the units row
    ours = df[df["Name"].str.contains("cosmaSgemm", na=False)]["Duration"].astype(float)
    assert list(ours) == [7.25]


def test_parse_rows():
    assert list(runner.parse_rows("", 3)) == [0, 1, 2]
    assert list(runner.parse_rows("1:10:4", 10)) == [1, 5, 9]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["native", "bf16x6"])
def test_runner_end_to_end(cuda, tmp_path, precision):
    lst = write_list(tmp_path)
    out = tmp_path / "runs"
    rows = ""  # the double row is skipped (noted in results.csv) on the FP32-only BF16 paths
    rc = runner.main([lst, "--out", str(out), "--runs", "3", "--warmup", "1", "--check", "--cublas",
                      "--precision", precision] + (["--rows", rows] if rows else []))
    assert rc == 0
    (d,) = os.listdir(out)
    files = sorted(os.listdir(out / d))
    assert "results.csv" in files
    assert sum(f.startswith("nvprof_") for f in files) == (4 if precision == "native" else 3)
    import pandas as pd

    res = pd.read_csv(out / d / "results.csv")
    ran = res[res["median_us"].notna()]
    assert len(ran) == (4 if precision == "native" else 3)
    assert ran["check_within_bound"].astype(bool).all()
    res = ran
    assert (res["median_us"] > 0).all()
