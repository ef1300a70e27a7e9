"""Copies the reference's golden fixtures used by the tests into tests/golden/.

The fixtures are the ``.npy`` arrays and ``meta.json`` files that
jmdelouis/STL-Dev-MPI commits under ``fixtures/`` (dumped from STL-Dev by its
``tools/dump_reference.py``); they pin the oracle.  Run once, in a checkout
that has the reference mounted:

    python tests/golden/collect.py /path/to/STL-Dev-MPI/fixtures

Without an argument the fixtures are read from $STL_REFERENCE_ROOT/fixtures
(STL_REFERENCE_ROOT defaults to /root/reference).

Only a subset is copied, to keep the repository small: every stats case,
and per geometry kind the cases listed in ``SELECT`` below.
"""
import json
import os
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent

SELECT = {
    "stats": lambda c: True,
    "synthesis": lambda c: True,
    "block": lambda c: c["kind"] == "wavelet",
    "geometry": lambda c: (
        c["kind"] in ("rotation", "kernel_grid", "neighbours")
        or (c["kind"] in ("centres", "interp") and c["nside"] in (1, 8, 1024))
        or (c["kind"] == "ring2nest" and c["order"] in (1, 3, 10))
        or (c["kind"] == "conv" and c["kernel_sz"] == 5 and c["G"] == 4 and c["gauge"] == "cosmo")
        or (c["kind"] == "conv" and c["block_start"] in (0, 4864) and c["nside"] in (8, 32))
        or (c["kind"] == "down" and (c["nside"] <= 32 or c["name"].endswith(("_s0", "_s4194304", "_s12581888"))))
    ),
}


def main(src: Path):
    for suite, keep in SELECT.items():
        index = json.loads((src / suite / "index.json").read_text())
        chosen = [c for c in index if keep(c)]
        out = HERE / suite
        out.mkdir(parents=True, exist_ok=True)
        for c in chosen:
            dst = out / c["name"]
            if dst.exists():
                shutil.rmtree(dst)
            shutil.copytree(src / suite / c["name"], dst)
        (out / "index.json").write_text(json.dumps(chosen, indent=1))
        print(f"{suite}: {len(chosen)} of {len(index)} cases")


if __name__ == "__main__":
    root = Path(os.environ.get("STL_REFERENCE_ROOT", "/root/reference"))
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else root / "fixtures")
