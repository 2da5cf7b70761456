"""Extract the reference's own known-answer vectors for the hot path into JSON.

Reads the Rust test modules of idrees2516/lzx (as text; nothing is compiled or
run) and writes ``reference_kats.json`` beside this script:

* Goldilocks add/sub/mul KATs, ``crates/lattice-core/src/field.rs`` (the
  ``python_cross_validated_kats`` test),
* FIPS-202 SHA3-256 / SHAKE256 digests, ``crates/lattice-core/src/keccak.rs``
  (``sha3_256_kat`` / ``shake256_kat``),
* the Modulus32 constants, ``crates/lattice-ring/src/modulus.rs``.

Usage: python tests/golden/extract_reference_kats.py REFERENCE_ROOT
(or with the REFERENCE_ROOT environment variable set to the checkout).
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _fn_body(src: str, name: str) -> tuple[str, int]:
    m = re.search(r"fn\s+" + name + r"\s*\(", src)
    if not m:
        raise SystemExit(f"test fn {name} not found")
    start = src.index("{", m.end())
    depth = 0
    for i in range(start, len(src)):
        if src[i] == "{":
            depth += 1
        elif src[i] == "}":
            depth -= 1
            if depth == 0:
                return src[start:i + 1], src.count("\n", 0, m.start()) + 1
    raise SystemExit("unbalanced braces")


def _tuples(block: str):
    body = re.sub(r"\s+", "", block)
    return [tuple(int(x) for x in t.split(",")) for t in re.findall(r"\((\d+,\d+,\d+),?\)", body)]


def goldilocks_kats(root: str) -> dict:
    path = "crates/lattice-core/src/field.rs"
    src = open(os.path.join(root, path)).read()
    body, line = _fn_body(src, "python_cross_validated_kats")
    out = {"source": f"{path}:{line}"}
    for op in ("sub", "add", "mul"):
        m = re.search(op + r"_cases:\s*&\[\(u64,\s*u64,\s*u64\)\]\s*=\s*&\[(.*?)\];", body, re.S)
        out[op] = [list(t) for t in _tuples(m.group(1))]
    return out


def keccak_kats(root: str) -> dict:
    path = "crates/lattice-core/src/keccak.rs"
    src = open(os.path.join(root, path)).read()
    cases = []
    body, line = _fn_body(src, "sha3_256_kat")
    calls = re.findall(r"sha3_256\((b\"[^\"]*\"|&\[0u8;\s*(\d+)\])\)", body)
    digests = re.findall(r"\"([0-9a-f]{64})\"", body)
    for (arg, zeros), dig in zip(calls, digests):
        msg = "00" * int(zeros) if zeros else arg[2:-1].encode().hex()
        cases.append({"fn": "sha3_256", "msg_hex": msg, "digest_hex": dig,
                      "source": f"{path}:{line}"})
    body, line = _fn_body(src, "shake256_kat")
    m = re.search(r"shake256\(b\"([^\"]*)\",\s*(\d+)\)", body)
    dig = re.search(r"\"([0-9a-f]{64})\"", body).group(1)
    cases.append({"fn": "shake256", "msg_hex": m.group(1).encode().hex(),
                  "out_len": int(m.group(2)), "digest_hex": dig, "source": f"{path}:{line}"})
    return {"cases": cases}


def modulus_constants(root: str) -> dict:
    path = "crates/lattice-ring/src/modulus.rs"
    src = open(os.path.join(root, path)).read()
    out = {}
    for name, q, a, g in re.findall(
            r"pub const (Q_\w+): Modulus32 = Modulus32::new\((\d+),\s*(\d+),\s*(\d+)\)", src):
        out[name] = {"q": int(q), "two_adicity": int(a), "generator": int(g)}
    out["source"] = path
    return out


def main() -> None:
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT")
    if not root:
        sys.exit("usage: extract_reference_kats.py REFERENCE_ROOT (or set REFERENCE_ROOT)")
    data = {
        "reference": "idrees2516/lzx",
        "goldilocks": goldilocks_kats(root),
        "keccak": keccak_kats(root),
        "modulus32": modulus_constants(root),
    }
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")
    print("wrote", os.path.join(HERE, "reference_kats.json"))


if __name__ == "__main__":
    main()
