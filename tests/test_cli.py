"""The command line stand-in: argument validation and error text as the
reference's pystamps-native parses them (pystamps-native.rs:216-345), with
the cuda kernel backend added; patch discovery as discover_dataset
(crates/pystamps-core/src/lib.rs:296-361). No GPU work here."""
import json
from pathlib import Path

import pytest

from pystamps_b200 import __main__ as cli


def test_kernel_backend_cuda_accepted_and_allowed_native_only():
    req, rt = cli.parse_run_args(["--dataset", "/d", "--native-only", "--backend", "native",
                                  "--stage2-kernel-backend", "CUDA", "--stage2-native-threads", "4"])
    assert rt["stage2_kernel_backend"] == "cuda" and rt["native_only"] and req["dataset_root"] == "/d"
    assert cli.parse_run_args(["--dataset", "x", "--stage2-kernel-backend", "gpu"])[1]["stage2_kernel_backend"] == "cuda"


@pytest.mark.parametrize("args,msg", [
    (["--stage2-kernel-backend", "cuda"], "expected --dataset PATH"),
    (["--dataset"], "expected --dataset PATH"),
    (["--dataset", "d", "--stage2-kernel-backend", "tpu"], "unsupported stage-2 kernel backend 'tpu'"),
    (["--dataset", "d", "--backend", "mpi"], "unsupported runtime backend 'mpi'"),
    (["--dataset", "d", "--native-only"], "native-only mode requires --backend native; got 'auto'"),
    (["--dataset", "d", "--native-only", "--backend", "native", "--stage2-kernel-backend", "python"],
     "native-only mode requires --stage2-kernel-backend native or cuda; got 'python'"),
    (["--dataset", "d", "--stage2-kernel-backend", "python", "--stage2-native-threads", "2"],
     "stage2-native-threads requires stage2 kernel backend auto or native"),
    (["--dataset", "d", "--start-step", "x"], "invalid --start-step value 'x': invalid digit found in string"),
    (["--dataset", "d", "--io-workers", "70000"], "invalid --io-workers value '70000': number too large"),
    (["--dataset", "d", "--bogus"], "unexpected run argument '--bogus'"),
])
def test_run_argument_errors(args, msg):
    with pytest.raises(cli.CliError, match=msg.replace("(", r"\(")):
        cli.parse_run_args(args)


def test_main_error_exit_and_text(capsys):
    assert cli.main(["stage2", "--patch"]) == 2
    assert "error: expected --patch PATH" in capsys.readouterr().err
    assert cli.main([]) == 2
    assert "error: missing subcommand" in capsys.readouterr().err
    assert cli.main(["stage9"]) == 2
    assert "unknown subcommand 'stage9'" in capsys.readouterr().err


def test_discovery_and_dry_run(tmp_path: Path, capsys):
    for n in ("PATCH_10", "PATCH_2", "PATCH_1", "other"):
        (tmp_path / n).mkdir()
    assert [p.name for p in cli.discover_patches(tmp_path)] == ["PATCH_1", "PATCH_2", "PATCH_10"]
    (tmp_path / "patch.list").write_text("# chosen\nPATCH_2\n\nPATCH_1\n")
    assert [p.name for p in cli.discover_patches(tmp_path)] == ["PATCH_2", "PATCH_1"]
    assert cli.main(["run", "--dataset", str(tmp_path), "--start-step", "2", "--end-step", "3", "--dry-run",
                     "--stage2-kernel-backend", "cuda"]) == 0
    out = json.loads(capsys.readouterr().out)
    assert [(r["stage"], r["target"], r["status"]) for r in out] == [
        (2, "PATCH_2", "pending_execution"), (2, "PATCH_1", "pending_execution"),
        (3, "PATCH_2", "skipped"), (3, "PATCH_1", "skipped")]
    with pytest.raises(cli.CliError, match="dataset does not exist"):
        cli.discover_patches(tmp_path / "nope")
    with pytest.raises(cli.CliError, match="invalid stage range 3..2; expected 1..8"):
        cli.execute_run({"dataset_root": str(tmp_path), "start_step": 3, "end_step": 2, "dry_run": True}, {})
