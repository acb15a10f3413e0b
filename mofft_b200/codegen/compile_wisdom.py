"""Compile the B200 plan wisdom JSON into the device plan cache table.

The B200 analogue of the reference's tools/compile_wisdom.py:12-157, which
turns plan-search JSON into the C lookup ``mofft_generated_wisdom_lookup``.
Input: ``mofft_b200/wisdom/b200_wisdom.json``::

    {"source": "...", "formal": false,
     "entries": [{"length": 4096, "precision_bits": 32,
                  "chain": [16, 16, 16],
                  "kernels": ["rows_float_4096_t256_b1_sfalse"]}, ...]}

``chain`` is the in-CTA Stockham stage list, first stage first (the
reference's radix chain reversed); ``kernels`` (optional) names the tuned
kernel instance of each pass among the variants that share a chain.  Entries are validated: the chain must
multiply to the length and use only radices of the reference's set.

Run: python -m mofft_b200.codegen.compile_wisdom [json] [out_header]
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

RADICES = {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 32, 64}
ROOT = Path(__file__).resolve().parents[1]


def load_entries(path: Path) -> tuple[list[dict], str, bool]:
    if not path.exists():
        return [], "none", False
    data = json.loads(path.read_text())
    entries = []
    seen = set()
    for e in data.get("entries", []):
        length = int(e["length"])
        bits = int(e["precision_bits"])
        chain = [int(r) for r in e["chain"]]
        if bits not in (32, 64):
            raise ValueError(f"bad precision in {e}")
        prod = 1
        for r in chain:
            if r not in RADICES:
                raise ValueError(f"unsupported radix {r} in {e}")
            prod *= r
        if prod != length or not 1 <= len(chain) <= 24:
            raise ValueError(f"chain does not multiply to length in {e}")
        key = (length, bits)
        if key in seen:
            raise ValueError(f"duplicate wisdom entry {key}")
        seen.add(key)
        kernels = [str(k) for k in e.get("kernels", [])][:4]
        entries.append({"length": length, "bits": bits, "chain": chain, "kernels": kernels})
    entries.sort(key=lambda e: (e["bits"], e["length"]))
    return entries, str(data.get("source", "unknown")), bool(data.get("formal", False))


def render(entries: list[dict], source: str, formal: bool) -> str:
    lines = [
        "/* Generated by mofft_b200/codegen/compile_wisdom.py -- do not edit. */",
        "#pragma once",
        "#include <stddef.h>",
        "typedef struct { size_t length; int precision_bits; int count; int chain[24];"
        " const char *kernels[4]; } mofft_wisdom_entry;",
        "static const mofft_wisdom_entry k_mofft_wisdom[] = {",
    ]
    for e in entries:
        chain = ", ".join(str(r) for r in e["chain"])
        names = ", ".join(f'"{k}"' for k in e["kernels"]) or "0"
        lines.append(f"  {{{e['length']}u, {e['bits']}, {len(e['chain'])}, {{{chain}}}, "
                     f"{{{names}}}}},")
    lines.append("  {0u, 0, 0, {0}, {0}},")
    lines.append("};")
    lines.append(f"#define MOFFT_WISDOM_COUNT {len(entries)}")
    lines.append(f"#define MOFFT_WISDOM_FORMAL {1 if formal else 0}")
    src = source.replace("\\", "\\\\").replace('"', '\\"')
    lines.append(f'#define MOFFT_WISDOM_SOURCE "{src}"')
    return "\n".join(lines) + "\n"


def main(argv: list[str]) -> int:
    src = Path(argv[1]) if len(argv) > 1 else ROOT / "wisdom" / "b200_wisdom.json"
    out = Path(argv[2]) if len(argv) > 2 else ROOT / "csrc" / "generated" / "wisdom_table.h"
    entries, source, formal = load_entries(src)
    text = render(entries, source, formal)
    out.parent.mkdir(parents=True, exist_ok=True)
    if not out.exists() or out.read_text() != text:
        out.write_text(text)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
