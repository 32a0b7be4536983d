"""The DRAM traffic that bench.py reports for the update kernel (`roofline.traffic`)
is a per-form constant taken from an ncu capture; each constant names the summary
under profiles/ that it comes from. These host tests keep the two in step: the
constant must equal that summary's `dram__bytes_read.sum + dram__bytes_write.sum`
(to the summary's printed precision), and every summary that bench.py cites must
exist."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _traffic_constants():
    src = open(os.path.join(ROOT, "bench.py")).read()
    block = src[src.index("NCU_TRAFFIC = {"):]
    block = block[:block.index("\n}\n")]
    pattern = re.compile(r'"(\w+)": \(([\d_]+) \+ ([\d_]+),\s*"[^"]*?(profiles/[\w.]+\.md)"\)', re.S)
    return [(m.group(1), int(m.group(2).replace("_", "")), int(m.group(3).replace("_", "")), m.group(4))
            for m in pattern.finditer(block)]


def _dram_mbytes(path, which):
    text = open(os.path.join(ROOT, path)).read()
    m = re.search(r"\| DRAM %s \(`dram__bytes_%s\.sum`\) \| ([\d.]+) Mbyte \|" % (which, which), text)
    assert m, f"{path} has no DRAM {which} line"
    digits = len(m.group(1).split(".")[1]) if "." in m.group(1) else 0
    return float(m.group(1)), digits


def test_every_update_form_has_a_traffic_constant():
    forms = {name for name, _, _, _ in _traffic_constants()}
    assert forms == {"dense", "sparse", "sparse_bf16"}


def test_traffic_constants_match_their_profiles():
    for name, read, write, path in _traffic_constants():
        assert os.path.exists(os.path.join(ROOT, path)), path
        for value, which in ((read, "read"), (write, "write")):
            mbytes, digits = _dram_mbytes(path, which)
            # the summary prints Mbyte with `digits` decimals
            assert abs(value / 1e6 - mbytes) <= 0.5 * 10.0 ** -digits + 1e-9, (name, which, value, mbytes)
