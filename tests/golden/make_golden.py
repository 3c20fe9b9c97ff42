"""Extracts the reference's own known answers from its sources, read as text,
into reference_facts.json beside this script, which the oracle's tests read.

    python tests/golden/make_golden.py [path of the reference checkout]

The reference is a Rust workspace that can't be built here, so its unit and
property tests give these facts as source text:
- the SplitMix64 outputs of seed 0 (crates/einfold-testkit/src/rng.rs),
- the tile-visit counts of masked pipelines
  (crates/einfold-kernels/tests/pipeline_vs_sql.rs),
- the Bounds decline cases (crates/einfold-kernels/src/fused.rs, its tests),
- the long shared prefix of the key-sorting test
  (crates/einfold-kernels/src/discriminate.rs, its tests),
- the seeds and case counts of the four property tests
  (crates/einfold-kernels/tests/*.rs).
Each fact records the file and line it came from.
"""
import ast
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "reference_facts.json")


def _read(root, rel):
    with open(os.path.join(root, rel)) as f:
        return f.read()


def _line(text, pos):
    return text.count("\n", 0, pos) + 1


def _int_expr(s):
    """An integer expression of literals (`16 * 17 / 2`, `8 * 10`) as Rust's
    integer arithmetic computes it."""
    s = s.replace("_", "").strip()

    def ev(n):
        if isinstance(n, ast.Constant) and isinstance(n.value, int):
            return n.value
        if isinstance(n, ast.BinOp):
            a, b = ev(n.left), ev(n.right)
            if isinstance(n.op, ast.Add):
                return a + b
            if isinstance(n.op, ast.Sub):
                return a - b
            if isinstance(n.op, ast.Mult):
                return a * b
            if isinstance(n.op, ast.Div):
                return a // b
        raise ValueError(f"not an integer expression: {s}")

    return ev(ast.parse(s, mode="eval").body)


def _f64(s):
    s = s.strip().replace("_", "")
    special = {"f64::INFINITY": "inf", "f64::NEG_INFINITY": "-inf", "f64::NAN": "nan"}
    if s in special:
        return special[s]
    return float(s)


def splitmix(root):
    rel = "crates/einfold-testkit/src/rng.rs"
    text = _read(root, rel)
    m = re.search(r"fn seed_zero_gives_splitmix64s_reference_outputs\(\).*?\[(.*?)\]\s*\)", text, re.S)
    words = [int(w.replace("_", ""), 16) for w in re.findall(r"0x[0-9a-f_]+", m.group(1))]
    return {"outputs": words, "source": f"{rel}:{_line(text, m.start())}"}


def tile_counts(root):
    rel = "crates/einfold-kernels/tests/pipeline_vs_sql.rs"
    text = _read(root, rel)
    comparisons = {"GreaterOrEqual": "ge", "Greater": "gt", "LessOrEqual": "le", "Less": "lt"}
    out = []
    for fn in re.finditer(r"#\[test\]\s*fn (\w+)\(\) \{(.*?)\n\}", text, re.S):
        body = fn.group(2)
        masks = {}
        for let in re.finditer(r"let (\w+) = \[(.*?)\];", body, re.S):
            conds = re.findall(r"\(Comparison::(\w+), (-?\d+)\)", let.group(2))
            masks[let.group(1)] = [[comparisons[c], int(o)] for c, o in conds]
        for a in re.finditer(r"assert_eq!\(tiles_visited\(([^,]+), (None|Some\((\d+)\)), &(\w+)\), \(([^,]+), ([^)]+)\)\);",
                             body):
            out.append({"test": fn.group(1), "length": _int_expr(a.group(1)),
                        "batches": int(a.group(3)) if a.group(3) else None, "conditions": masks[a.group(4)],
                        "visited": _int_expr(a.group(5)), "tiles": _int_expr(a.group(6)),
                        "source": f"{rel}:{_line(text, fn.start(2) + a.start())}"})
    return out


def bounds_cases(root):
    rel = "crates/einfold-kernels/src/fused.rs"
    text = _read(root, rel)
    out = []
    pattern = (r"assert!\((!?)(normal|bounds)\(([^)]*)\)\.hold\((Some\(([^)]*)\)|None), &\[([^\]]*)\], "
               r"&\[([^\]]*)\]\)\);")
    for m in re.finditer(pattern, text):
        args = [_f64(x) for x in m.group(3).split(",")]
        if m.group(2) == "normal":
            heaviest, lightest, largest, smallest = args
        else:  # bounds(heaviest, largest): lightest the least subnormal, smallest = largest
            heaviest, largest = args
            lightest, smallest = 5e-324, largest
        out.append({"holds": m.group(1) == "", "heaviest": heaviest, "lightest": lightest, "largest": largest,
                    "smallest": smallest, "terms": 3,
                    "z": _f64(m.group(5)) if m.group(5) is not None else None,
                    "results": [_f64(x) for x in m.group(6).split(",")],
                    "special": [x.strip() == "true" for x in m.group(7).split(",")],
                    "source": f"{rel}:{_line(text, m.start())}"})
    # The helpers' fixed fields, checked rather than assumed.
    assert re.search(r"fn bounds\(heaviest: f64, largest: f64\) -> Bounds \{\s*Bounds \{\s*heaviest,\s*"
                     r"lightest: f64::from_bits\(1\),\s*largest,\s*smallest: largest,\s*terms: 3,", text), \
        "bounds() changed"
    assert re.search(r"fn normal\(heaviest: f64, lightest: f64, largest: f64, smallest: f64\) -> Bounds \{"
                     r"\s*Bounds \{\s*heaviest,\s*lightest,\s*largest,\s*smallest,\s*terms: 3,", text), "normal() changed"
    return out


def long_prefix(root):
    rel = "crates/einfold-kernels/src/discriminate.rs"
    text = _read(root, rel)
    m = re.search(r'let prefix = "(\w)"\.repeat\(([\d_]+)\);\s*let strings: Vec<String> = \(0\.\.(\d+)\)\.rev\(\)'
                  r'\.map\(\|i\| format!\("\{prefix\}\{i:0(\d)\}"\)\)', text)
    return {"char": m.group(1), "prefix_bytes": int(m.group(2).replace("_", "")), "keys": int(m.group(3)),
            "digits": int(m.group(4)), "order": "reversed", "source": f"{rel}:{_line(text, m.start())}"}


def property_tests(root):
    out = {}
    for name in ("kernels_vs_sql", "pipeline_vs_sql", "expression_vs_sql"):
        rel = f"crates/einfold-kernels/tests/{name}.rs"
        text = _read(root, rel)
        s = re.search(r"\.unwrap_or\((0x[0-9a-f_]+)\);", text)
        c = re.search(r"Err\(_\) => (\d+),", text)
        out[name] = {"seed": int(s.group(1).replace("_", ""), 16), "cases": int(c.group(1)),
                     "source": f"{rel}:{_line(text, s.start())}"}
    rel = "crates/einfold-kernels/tests/dense_metamorphic.rs"
    text = _read(root, rel)
    s = re.search(r'env\("EINFOLD_SEED"\)\.unwrap_or\((0x[0-9a-f_]+)\);', text)
    c = re.search(r'env\("EINFOLD_CASES"\)\.unwrap_or\((\d+)\)', text)
    out["dense_metamorphic"] = {"seed": int(s.group(1).replace("_", ""), 16), "cases": int(c.group(1)),
                                "source": f"{rel}:{_line(text, s.start())}"}
    return out


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    facts = {"splitmix64_seed0": splitmix(root), "tile_counts": tile_counts(root),
             "bounds_cases": bounds_cases(root), "long_prefix": long_prefix(root),
             "property_tests": property_tests(root)}
    with open(OUT, "w") as f:
        json.dump(facts, f, indent=1)
        f.write("\n")
    print(f"{OUT}: {len(facts['tile_counts'])} tile counts, {len(facts['bounds_cases'])} Bounds cases")


if __name__ == "__main__":
    main()
