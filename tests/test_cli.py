"""The reference-compatible command line (flagfft_b200.cli): option parsing,
argument checks and report shapes of `flagfft-cli bench`
(src/cli_tools/flagfft-cli/main.cpp:46-133, src/cli_tools/bench/report.cpp:
12-67) on the CPU; one case end to end on the GPU."""
import json

import pytest

from flagfft_b200 import cli


def test_defaults_and_shapes():
    a = cli.parse_bench_args([])
    assert a["warmup"] == 10 and a["iters"] == 100 and not a["json"]
    c = a["cases"][0]
    assert (c.api, c.shape, c.batch, c.direction, c.placement, c.rank) == ("c2c", [16], 1, -1, "out-of-place", 1)
    a = cli.parse_bench_args(["--rank", "2", "--shape", "64x32,128x16", "--api", "z2z", "--batch", "3",
                              "--direction", "inv", "--placement", "in-place", "--json", "--print-path"])
    assert [c.shape for c in a["cases"]] == [[64, 32], [128, 16]]
    assert all(c.direction == 1 and c.placement == "in-place" and c.batch == 3 for c in a["cases"])
    assert a["json"] and a["print_path"]


@pytest.mark.parametrize("argv,msg", [
    (["--rank", "4"], "invalid --rank"),
    (["--rank", "2", "--shape", "16x16", "--api", "r2c"], "rank 2 currently supports only c2c and z2z"),
    (["--rank", "3", "--shape", "8x8x8", "--batch", "2"], "--batch is only supported"),
    (["--rank", "2", "--shape", "16"], "dimension count"),
    (["--api", "r2c", "--direction", "inverse"], "only supports forward"),
    (["--api", "z2d"], "only supports inverse"),
    (["--batch", "0"], "must be positive"),
    (["--frobnicate"], "unknown argument"),
    (["--iters"], "requires a value"),
])
def test_argument_checks(argv, msg):
    with pytest.raises(cli.CliError) as e:
        cli.parse_bench_args(argv)
    assert msg in str(e.value)


def test_percentile_and_reports():
    assert cli.percentile([5.0, 1.0, 3.0, 2.0, 4.0], 0.5) == 3.0
    assert cli.percentile([5.0, 1.0, 3.0, 2.0, 4.0], 0.9) == 5.0
    cases = cli.parse_bench_args(["--shape", "4096", "--batch", "256"])["cases"]
    res = [{"flagfft_median_ms": 0.01, "flagfft_p90_ms": 0.012, "ref_median_ms": 0.02, "ref_p90_ms": 0.021,
            "speedup": 2.0, "plan_description": "tree"}]
    j = cli.format_json(cases, res, 10, 100)
    assert j["status"] == "passed" and j["command"] == "bench"
    e = j["cases"][0]
    assert e["api"] == "c2c" and e["shape"] == [4096] and e["rank"] == 1 and e["batch"] == 256
    assert e["direction"] == "forward" and e["placement"] == "out-of-place" and e["plan_description"] == "tree"
    assert set(e["timing"]) == {"flagfft_median_ms", "flagfft_p90_ms", "ref_median_ms", "ref_p90_ms", "speedup",
                                "warmup", "iters"}
    table = cli.format_table(cases, res, 10, 100)
    assert table.splitlines()[0].startswith("shape") and "2.00x" in table


def test_main_usage_and_errors(capsys):
    assert cli.main(["--help"]) == 0
    assert cli.main(["frob"]) == cli.EXIT_USAGE
    assert cli.main(["bench", "--rank", "9"]) == cli.EXIT_FAILED


@pytest.mark.gpu
@pytest.mark.parametrize("argv", [["--shape", "4096", "--batch", "64"], ["--api", "r2c", "--shape", "1000"],
                                  ["--api", "z2d", "--direction", "inverse", "--shape", "1024",
                                   "--placement", "in-place"],
                                  ["--rank", "2", "--shape", "64x128", "--api", "c2c", "--batch", "2"]])
def test_bench_end_to_end(torch_cuda, capsys, argv):
    assert cli.main(["bench", *argv, "--warmup", "2", "--iters", "6", "--json", "--print-path"]) == 0
    out = json.loads(capsys.readouterr().out)
    t = out["cases"][0]["timing"]
    assert t["flagfft_median_ms"] > 0 and t["ref_median_ms"] > 0 and t["iters"] == 6
    assert "Plan tree" in out["cases"][0]["plan_description"]
