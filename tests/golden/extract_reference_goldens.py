"""Extract the golden values of the reference's host tests into ``reference_goldens.json``.

Reads the reference's ``test/test.cpp`` as text (nothing is compiled or run) and records:

* every ``EXPECT_FLOAT_EQ(<expr>, <arithmetic of numeric literals>)`` with its line number, the
  enclosing test name and the literal value (e.g. ``test/test.cpp:59`` -> 0.03846154);
* every ``std::vector<float> expected = { ... }`` block (the D1/D2/D3 random diffusion goldens).

The parity tests look golden values up by ``file:line`` so each check cites where its number
comes from.  Regenerate with::

    python tests/golden/extract_reference_goldens.py /path/to/paraBioFVM
"""

from __future__ import annotations

import ast
import json
import operator
import os
import re
import sys

_OPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv}


def _eval_literal_arith(text: str):
    """Evaluate +,-,*,/ over numeric literals; None if the text is anything else."""
    text = text.strip().rstrip("f")
    text = re.sub(r"(\d)\.(?=\D|$)", r"\1.0", text)  # "20." -> "20.0"
    try:
        node = ast.parse(text, mode="eval").body
    except SyntaxError:
        return None

    def ev(n):
        if isinstance(n, ast.Constant) and isinstance(n.value, (int, float)):
            return float(n.value)
        if isinstance(n, ast.UnaryOp) and isinstance(n.op, (ast.USub, ast.UAdd)):
            v = ev(n.operand)
            return -v if isinstance(n.op, ast.USub) else v
        if isinstance(n, ast.BinOp) and type(n.op) in _OPS:
            return _OPS[type(n.op)](ev(n.left), ev(n.right))
        raise ValueError

    try:
        return ev(node)
    except (ValueError, ZeroDivisionError):
        return None


def _split_top_level_comma(args: str):
    depth = 0
    for i, ch in enumerate(args):
        if ch in "(<{[":
            depth += 1
        elif ch in ")>}]":
            depth -= 1
        elif ch == "," and depth == 0:
            return args[:i], args[i + 1:]
    return None


def extract(ref_root: str) -> dict:
    path = os.path.join(ref_root, "test", "test.cpp")
    with open(path) as f:
        lines = f.read().split("\n")

    scalars = {}
    vectors = {}
    test_name = None
    test_re = re.compile(r"^\s*TEST(?:_P)?\(\s*(\w+)\s*,\s*(\w+)\s*\)")
    for ln, line in enumerate(lines, start=1):
        m = test_re.match(line)
        if m:
            test_name = f"{m.group(1)}.{m.group(2)}"
        if "EXPECT_FLOAT_EQ(" in line:
            # join continuation lines until the parentheses balance
            text = line
            k = ln
            while text.count("(") > text.count(")") and k < len(lines):
                text += " " + lines[k].strip()
                k += 1
            inner = text[text.index("EXPECT_FLOAT_EQ(") + len("EXPECT_FLOAT_EQ("):]
            inner = inner[: inner.rindex(")")].replace("->", ".")
            parts = _split_top_level_comma(inner)
            if not parts:
                continue
            value = _eval_literal_arith(parts[1])
            if value is None:
                continue
            scalars[str(ln)] = {"test": test_name, "expr": " ".join(parts[0].split()), "value": value}
        if re.search(r"std::vector<float>\s+expected\s*=\s*\{", line):
            body = ""
            k = ln - 1
            while True:
                body += lines[k]
                if "}" in lines[k]:
                    break
                k += 1
            nums = body[body.index("{") + 1: body.index("}")]
            vectors[test_name] = {"line": ln, "values": [float(t) for t in nums.replace("\t", " ").split(",") if t.strip()]}

    return {
        "source": "test/test.cpp of asmelko/paraBioFVM (read as text)",
        "scalars": {"test/test.cpp": scalars},
        "vectors": vectors,
    }


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: extract_reference_goldens.py <paraBioFVM source root>")
    ref_root = sys.argv[1]
    data = extract(ref_root)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_goldens.json")
    with open(out, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    n = len(data["scalars"]["test/test.cpp"])
    print(f"wrote {out}: {n} scalar goldens, {len(data['vectors'])} vectors")


if __name__ == "__main__":
    main()
