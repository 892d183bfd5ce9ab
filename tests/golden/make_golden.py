"""Generate the golden fixtures that pin the spin tables and the UDSC sparse
lists against the reference.

Run in a container where the PLEGMA sources are mounted (default path below);
it reads the reference's own tables as text and stores only their SHA-256
digests (tests/golden/ref_table_digests.json), so no reference table is copied
into this repository.  The tests recompute the digests from the tables that
plegma_b200.spin derives from the gamma-matrix definitions.

    python tests/golden/make_golden.py [/path/to/PLEGMA]
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from plegma_b200 import spin  # noqa: E402


def c_array_numbers(text: str, name: str):
    """Numbers of the brace initialiser that follows `name[...] =`."""
    m = re.search(re.escape(name) + r"\s*(\[[^=]*\])\s*=\s*\{", text)
    if not m:
        raise KeyError(name)
    i = m.end() - 1
    depth = 0
    j = i
    while True:
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                break
        j += 1
    body = re.sub(r"//[^\n]*", "", text[i:j + 1])
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    return [float(x) for x in re.findall(r"-?\d+(?:\.\d+)?(?:[eE][-+]?\d+)?", body)]


def reference_digests(ref_root: str):
    kern = os.path.join(ref_root, "lib", "kernels")
    with open(os.path.join(kern, "PLEGMA_gammas.cuh")) as f:
        gam = f.read()
    with open(os.path.join(kern, "PLEGMA_baryons_NtoN.cu")) as f:
        nton = f.read()
    with open(os.path.join(kern, "PLEGMA_baryons_deltas.cu")) as f:
        dl = f.read()
    with open(os.path.join(kern, "PLEGMA_kernel_utils.cuh")) as f:
        ku = f.read()
    g_val = c_array_numbers(gam, "gamma")           # [16][4][2] (re, im)
    g_ind = c_array_numbers(gam, "gammaInd")        # [16][4][2] (row, col)
    out = {
        "gamma_values": spin.table_digest(g_val),
        "gamma_indices": spin.table_digest(g_ind),
        "nucleon_indices": spin.table_digest(c_array_numbers(nton, "NtoN_indices")),
        "nucleon_values": spin.table_digest(c_array_numbers(nton, "NtoN_values")),
        "delta_indices": spin.table_digest(c_array_numbers(dl, "deltas_indices")),
        "delta_values": spin.table_digest(c_array_numbers(dl, "deltas_values")),
        "eps": spin.table_digest(c_array_numbers(ku, "eps")),
        "sgn_eps": spin.table_digest(c_array_numbers(ku, "sgn_eps")),
    }
    for key, fname, tname in (("ntor", "PLEGMA_baryons_NtoR.cu", "NTR"), ("rton", "PLEGMA_baryons_RtoN.cu", "RtoN"),
                              ("rtor", "PLEGMA_baryons_RtoR.cu", "RTR")):
        with open(os.path.join(kern, fname)) as f:
            src = f.read()
        out[key + "_indices"] = spin.table_digest(c_array_numbers(src, tname + "_indices"))
        out[key + "_values"] = spin.table_digest(c_array_numbers(src, tname + "_values"))
    out.update(reference_udsc_digests(kern))
    return out


def reference_udsc_digests(kern: str):
    """Digests of the reference's table-driven baryon lists
    (PLEGMA_baryons_udsc_arrays.cu/.cuh, written by its python/baryons.py):
    the product list, the dataset names, and per dataset the ordered
    (6 spin indices, single-precision weight) entries."""
    from plegma_b200 import udsc
    with open(os.path.join(kern, "PLEGMA_baryons_udsc_arrays.cuh")) as f:
        hdr = f.read()
    with open(os.path.join(kern, "PLEGMA_baryons_udsc_arrays.cu")) as f:
        arr = f.read()
    prods = re.findall(r'"(\w+)"', re.search(r"BP_prop_prods\s*=\s*\{(.*?)\};", hdr).group(1))
    names_block = re.search(r"BP_prop_prods_names\s*=\s*\{(.*?)\};\n", hdr, flags=re.S).group(1)
    names = re.findall(r'"([^"]+)"', names_block)
    out = {"udsc_products": udsc.names_digest(prods), "udsc_names": udsc.names_digest(names)}
    ds = {}
    for n in names:
        key = n.replace("/", "_")
        idx = [int(x) for x in c_array_numbers(arr, key + "_idxs")]
        vals = c_array_numbers(arr, key + "_vals")
        tups = [tuple(idx[6 * i:6 * i + 6]) for i in range(len(idx) // 6)]
        w = [complex(vals[2 * i], vals[2 * i + 1]) for i in range(len(vals) // 2)]
        ds[n] = udsc.ordered_digest(tups, w)
    out["udsc_datasets"] = ds
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PLEGMA_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set PLEGMA_REFERENCE)")
    digests = reference_digests(ref)
    path = os.path.join(HERE, "ref_table_digests.json")
    with open(path, "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
