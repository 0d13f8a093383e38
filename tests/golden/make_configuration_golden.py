"""Extracts the configuration-signature golden values from the reference's own test,
ConfigurationTest.java, into configuration_golden.json (committed).

    python tests/golden/make_configuration_golden.py /path/to/reference

For each configuration of the test (spi in cycle notation, pi = (0 1 ... n-1)) it records
the signature, the canonical signature, the hash code and the set of equivalent signatures
the test asserts.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_floats(text):
    return [float(t.rstrip("f")) for t in re.findall(r"-?\d+\.\d+f?", text)]


def main(ref_root):
    path = os.path.join(ref_root, "src/test/java/br/unb/cic/tdp/base/ConfigurationTest.java")
    src = open(path).read()
    out = {}
    # each block starts with a "// Configuration k: (...)" banner
    banners = list(re.finditer(r"// Configuration \d+: (\([^\n]*\))", src))
    for b, m in enumerate(banners):
        spi = m.group(1).strip()
        block = src[m.end(): banners[b + 1].start() if b + 1 < len(banners) else len(src)]
        rec = {"spi": spi}
        sig = re.search(r"void testConfig\d+_Signature\(\).*?expectedSignature = \{([^}]*)\}", block, re.S)
        can = re.search(r"expectedCanonicalSignature = \{([^}]*)\}", block, re.S)
        hc = re.search(r"assertEquals\((-?\d+), config\.hashCode\(\)\)", block)
        eq = re.search(r"expectedSignatures = Arrays\.asList\((.*?)\);", block, re.S)
        if sig:
            rec["signature"] = parse_floats(sig.group(1))
        if can:
            rec["canonical_signature"] = parse_floats(can.group(1))
        if hc:
            rec["hash_code"] = int(hc.group(1))
        if eq:
            rec["equivalent_signatures"] = [parse_floats(s) for s in re.findall(r'"\[([^\]]*)\]"', eq.group(1))]
        out[spi] = rec
    dst = os.path.join(HERE, "configuration_golden.json")
    with open(dst, "w") as fh:
        json.dump({"source": "src/test/java/br/unb/cic/tdp/base/ConfigurationTest.java",
                   "configurations": list(out.values())}, fh, indent=1)
    print(f"wrote {dst}: {len(out)} configurations")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(f"usage: python {sys.argv[0]} <reference checkout>")
    main(sys.argv[1])
