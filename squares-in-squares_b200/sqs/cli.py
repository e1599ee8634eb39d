"""Command line tools of the reference's `squares` program (cli.py:29-130)
on the GPU certifier and annealer:

    python -m sqs.cli baseline --max-n N --output submission.csv
    python -m sqs.cli validate INPUT [--max-n N] [--report R] [--require-complete]
    python -m sqs.cli score INPUT [--max-n N] [--report R]
    python -m sqs.cli export-kaggle INPUT --output OUT
    python -m sqs.cli merge INPUT... --output OUT
    python -m sqs.cli optimize --n N [--input CSV] [--attempts A] [--maxiter M] [--seed S] --output OUT

Same arguments, the same JSON summary on stdout (the full report with
per-n results to --report), exit status 2 with "error: ..." on a
ValueError, KeyError or OSError.  (The reference's `references` command,
which imports credited record files, is not part of this library.)
"""
from __future__ import annotations

import argparse
import json
from pathlib import Path

from . import core


def bounded_n(value: str) -> int:
    n = int(value)
    if not 1 <= n <= 1000:
        raise argparse.ArgumentTypeError("must be in 1..1000")
    return n


def emit(report: dict, path: str | None = None) -> None:
    text = json.dumps(report, indent=2) + "\n"
    if path:
        target = Path(path)
        target.parent.mkdir(parents=True, exist_ok=True)
        target.write_text(text, encoding="utf-8")
    print(json.dumps({k: v for k, v in report.items() if k != "results"}, indent=2))


def main(argv: list[str] | None = None) -> None:
    parser = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    commands = parser.add_subparsers(dest="command", required=True)
    baseline = commands.add_parser("baseline", help="exact grid for n=1..max-n")
    baseline.add_argument("--max-n", type=bounded_n, default=1000)
    baseline.add_argument("--output", default="submission.csv")
    for name in ("validate", "score"):
        c = commands.add_parser(name)
        c.add_argument("input")
        c.add_argument("--max-n", type=bounded_n, default=1000)
        c.add_argument("--report")
        if name == "validate":
            c.add_argument("--require-complete", action="store_true")
    export = commands.add_parser("export-kaggle", help="open contact gaps and certify the numeric transport")
    export.add_argument("input")
    export.add_argument("--output", required=True)
    merge = commands.add_parser("merge", help="certified best side per n")
    merge.add_argument("inputs", nargs="+")
    merge.add_argument("--output", required=True)
    opt = commands.add_parser("optimize", help="certified GPU search for one n")
    opt.add_argument("--n", type=bounded_n, required=True)
    opt.add_argument("--input", help="optional CSV warm start")
    opt.add_argument("--attempts", type=int, default=20)
    opt.add_argument("--maxiter", type=int, default=250)
    opt.add_argument("--seed", type=int, default=42)
    opt.add_argument("--output", required=True)
    args = parser.parse_args(argv)
    try:
        if args.command == "baseline":
            puzzles = {n: core.grid(n) for n in range(1, args.max_n + 1)}
            core.write_submission(args.output, puzzles, validate=False)
            emit(dict(output=args.output, puzzles=args.max_n, rows=sum(len(r) for r in puzzles.values()),
                      score=sum(core.infeasible_score(n) for n in range(1, args.max_n + 1)),
                      certification="exact rational grid construction"))
        elif args.command in ("validate", "score"):
            puzzles = core.read_submission(args.input)
            if args.command == "validate":
                core.certify_all(puzzles)
                if args.require_complete and set(puzzles) != set(range(1, args.max_n + 1)):
                    raise ValueError("submission does not contain exactly 1..max-n")
            transported = core.kaggle_roundtrip(puzzles)
            if args.command == "validate":
                core.certify_all(transported)
            emit(core.score(transported, args.max_n), args.report)
        elif args.command == "export-kaggle":
            puzzles = core.prepare_kaggle(core.read_submission(args.input))
            core.write_submission(args.output, puzzles)
            emit(dict(output=args.output, puzzles=len(puzzles),
                      certification="interval certifier, decimal and numeric transport"))
        elif args.command == "merge":
            puzzles = core.merge_best([core.read_submission(p) for p in args.inputs])
            core.write_submission(args.output, puzzles)
            emit(dict(output=args.output, puzzles=len(puzzles)))
        elif args.command == "optimize":
            from .optimizer import optimize_packing
            initial = None
            if args.input:
                initial = core.read_submission(args.input).get(args.n)
                if initial is None:
                    raise ValueError(f"warm start has no n={args.n}")
            rows, report = optimize_packing(args.n, initial, attempts=args.attempts, seed=args.seed,
                                            maxiter=args.maxiter)
            core.write_submission(args.output, {args.n: rows})
            emit(report)
    except (ValueError, KeyError, OSError) as error:
        parser.exit(2, f"error: {error}\n")


if __name__ == "__main__":
    main()
