"""Command line stand-in for the reference's Rust stage-2 dispatch with the
``cuda`` kernel backend (the Rust toolchain is not available to build the
``pystamps-native`` binary itself).

    python -m pystamps_b200 stage2 --patch PATCH_DIR
    python -m pystamps_b200 run --dataset DATASET [--start-step 2] [--end-step 2]
        [--dry-run] [--native-only] [--backend native]
        [--stage2-kernel-backend cuda] [--stage2-native-threads N]

``run`` parses and validates its arguments as parse_run_args /
validate_runtime_config do (crates/pystamps-core/src/bin/pystamps-native.rs:
216-311), with ``cuda`` (alias ``gpu``) added to the stage-2 kernel backends
and allowed under ``--native-only`` (the change the drop-in makes at
:330-345). Patches are found as discover_dataset finds them
(crates/pystamps-core/src/lib.rs:296-361: ``patch.list`` or the PATCH_*
directories in numeric order). Stage 2 of each patch runs through
``stage2_estimate_gamma`` (run_native_stage (2, Patch), pystamps-native.rs:
198-201) and the per-patch results are printed as JSON like
execute_run_pipeline (:149-180). Steps other than 2 are outside this library
and are reported as skipped. Errors are printed as the reference prints them
("error: ..." and the usage text, exit status 2, pystamps-native.rs:63-72).
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

BACKENDS = {"auto": "auto", "threads": "threads", "thread": "threads", "io": "threads", "processes": "processes",
            "process": "processes", "cpu": "processes", "gpu": "gpu", "native": "native"}
KERNEL_BACKENDS = {"auto": "auto", "native": "native", "python": "python", "cpu": "python", "cuda": "cuda",
                   "gpu": "cuda"}

USAGE = ("usage: python -m pystamps_b200 stage2 --patch PATH\n"
         "       python -m pystamps_b200 run --dataset PATH [--start-step N] [--end-step N] [--dry-run] "
         "[--native-only] [--backend B] [--stage2-kernel-backend auto|native|python|cuda] "
         "[--io-workers N] [--cpu-workers N] [--stage2-native-threads N]")


class CliError(Exception):
    pass


def _value(args: list[str], ix: int, name: str) -> str:
    if ix + 1 >= len(args):
        raise CliError(f"{name} requires a value")
    return args[ix + 1]


def _unsigned(args: list[str], ix: int, name: str, top: int) -> int:
    """Rust's str::parse::<u8 / u16> with its error text."""
    v = _value(args, ix, name)
    if not v.isdigit():
        raise CliError(f"invalid {name} value '{v}': invalid digit found in string")
    if int(v) > top:
        raise CliError(f"invalid {name} value '{v}': number too large to fit in target type")
    return int(v)


def parse_run_args(args: list[str]) -> tuple[dict, dict]:
    """parse_run_args (pystamps-native.rs:216-282) + validate_runtime_config (:284-311)."""
    req = {"dataset_root": "", "start_step": 1, "end_step": 8, "dry_run": False}
    rt = {"native_only": False, "backend": "auto", "stage2_kernel_backend": "auto", "io_workers": 0,
          "cpu_workers": 0, "stage2_native_threads": 0}
    ix = 0
    while ix < len(args):
        a = args[ix]
        if a == "--dataset":
            if ix + 1 >= len(args):
                raise CliError("expected --dataset PATH")
            req["dataset_root"] = args[ix + 1]
            ix += 2
        elif a in ("--start-step", "--end-step"):
            req[a[2:].replace("-", "_")] = _unsigned(args, ix, a, 255)
            ix += 2
        elif a == "--dry-run":
            req["dry_run"] = True
            ix += 1
        elif a == "--native-only":
            rt["native_only"] = True
            ix += 1
        elif a == "--backend":
            v = _value(args, ix, a).lower()
            if v not in BACKENDS:
                raise CliError(f"unsupported runtime backend '{v}'")
            rt["backend"] = BACKENDS[v]
            ix += 2
        elif a == "--stage2-kernel-backend":
            v = _value(args, ix, a).lower()
            if v not in KERNEL_BACKENDS:
                raise CliError(f"unsupported stage-2 kernel backend '{v}'")
            rt["stage2_kernel_backend"] = KERNEL_BACKENDS[v]
            ix += 2
        elif a in ("--io-workers", "--cpu-workers", "--stage2-native-threads"):
            rt[a[2:].replace("-", "_")] = _unsigned(args, ix, a, 65535)
            ix += 2
        else:
            raise CliError(f"unexpected run argument '{a}'")
    if not req["dataset_root"]:
        raise CliError("expected --dataset PATH")
    validate_runtime_config(rt)
    return req, rt


def validate_runtime_config(rt: dict) -> None:
    backend, kb = rt["backend"], rt["stage2_kernel_backend"]
    if backend not in ("auto", "threads", "processes", "gpu", "native"):
        raise CliError(f"unsupported runtime backend '{backend}'")
    if kb not in ("auto", "python", "native", "cuda"):
        raise CliError(f"unsupported stage-2 kernel backend '{kb}'")
    if rt["stage2_native_threads"] > 0 and kb == "python":
        raise CliError("stage2-native-threads requires stage2 kernel backend auto or native")
    if rt["native_only"]:
        if backend != "native":
            raise CliError(f"native-only mode requires --backend native; got '{backend}'")
        if kb not in ("native", "cuda"):
            raise CliError(f"native-only mode requires --stage2-kernel-backend native or cuda; got '{kb}'")


def discover_patches(root: Path) -> list[Path]:
    """discover_dataset (crates/pystamps-core/src/lib.rs:296-361)."""
    if not root.exists():
        raise CliError(f"dataset does not exist: {root}")
    if not root.is_dir():
        raise CliError(f"dataset path is not a directory: {root}")
    plist = root / "patch.list"
    if plist.exists():
        out = []
        for name in (ln.strip() for ln in plist.read_text().splitlines()):
            if not name or name.startswith("#"):
                continue
            p = root / name
            if not (name.startswith("PATCH_") and "/" not in name and "\\" not in name) or not p.is_dir():
                raise CliError(f"dataset path is not a directory: {p}")
            out.append(p)
        if out:
            return out

    def key(p: Path):
        suffix = p.name[len("PATCH_"):]
        return (int(suffix) if suffix.isdigit() else 2 ** 64 - 1, p.name)

    return sorted((p for p in root.iterdir() if p.is_dir() and p.name.startswith("PATCH_")), key=key)


def run_stage2(patch: Path, kernel_backend: str = "cuda") -> str:
    from .stage2 import stage2_estimate_gamma

    if kernel_backend not in ("cuda", "auto"):
        raise CliError(f"stage-2 kernel backend '{kernel_backend}' is not provided by this library; use cuda")
    return stage2_estimate_gamma(patch, kernel_backend="cuda")


def execute_run(req: dict, rt: dict) -> list[dict]:
    s0, s1 = req["start_step"], req["end_step"]
    if s0 == 0 or s1 == 0 or s0 > s1 or s1 > 8:
        raise CliError(f"invalid stage range {s0}..{s1}; expected 1..8")
    patches = discover_patches(Path(req["dataset_root"]))
    results = []
    for stage in range(s0, s1 + 1):
        for patch in patches:
            r = {"stage": stage, "scope": "patch", "target": patch.name, "status": "pending_execution",
                 "details": "", "duration_sec": None}
            if stage != 2:
                r.update(status="skipped", details=f"stage {stage} is outside this library (stage 2 only)")
            elif not req["dry_run"]:
                t0 = time.perf_counter()
                try:
                    r.update(status="completed", details=run_stage2(patch, rt["stage2_kernel_backend"]))
                except Exception as err:  # the reference records the failure and carries on
                    r.update(status="failed", details=str(err))
                r["duration_sec"] = time.perf_counter() - t0
            results.append(r)
    return results


def main(argv: list[str] | None = None) -> int:
    args = list(sys.argv[1:] if argv is None else argv)
    try:
        if not args:
            raise CliError("missing subcommand")
        cmd, rest = args[0], args[1:]
        if cmd == "stage2":
            if len(rest) == 2 and rest[0] == "--patch":
                print(run_stage2(Path(rest[1])))
                return 0
            raise CliError("expected --patch PATH")
        if cmd == "run":
            req, rt = parse_run_args(rest)
            print(json.dumps(execute_run(req, rt), indent=2))
            return 0
        raise CliError(f"unknown subcommand '{cmd}'")
    except CliError as err:
        print(f"error: {err}", file=sys.stderr)
        print(USAGE, file=sys.stderr)
        return 2


if __name__ == "__main__":
    sys.exit(main())
