"""The table-driven baryon spin lists (plegma_b200/udsc.py) against the
reference's generated lists, through the digests that
tests/golden/make_golden.py computed from
lib/kernels/PLEGMA_baryons_udsc_arrays.{cuh,cu}: same products, same dataset
names in the same order, and per dataset the same (6 spin indices,
single-precision weight) entries in the same order."""
import json
import os

import numpy as np
import pytest

from plegma_b200 import udsc

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_table_digests.json")


@pytest.fixture(scope="module")
def gold():
    with open(GOLD) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def prods():
    return udsc.products()


def test_products_and_names_match_reference(gold, prods):
    assert udsc.names_digest([k for k, _ in prods]) == gold["udsc_products"]
    names = [n for _, dss in prods for n, _, _ in dss]
    assert udsc.names_digest(names) == gold["udsc_names"]
    assert len(names) == len(gold["udsc_datasets"]) == 200


def test_every_dataset_matches_reference(gold, prods):
    bad = [n for _, dss in prods for n, t, w in dss if udsc.ordered_digest(t, w) != gold["udsc_datasets"][n]]
    assert not bad, bad[:5]


def test_entry_counts_of_the_light_baryons(prods):
    d = {n: len(t) for _, dss in prods for n, t, _ in dss}
    assert d["proton/Pp_Cg5_Cg5"] == 56
    assert d["DeltaPl/Pp_Cgi_Cgi"] == 194
    assert d["DeltaPl/Ppgigj_Cgi_Cgj"] == 188
    assert d["DeltaPlPl/Pp_Cgi_Cgi"] == 112


def test_projectors_add_up_and_the_proton_is_real(prods):
    """P+ + P- = 1: the Pp and Pm lists of a baryon add up to the list of the
    unprojected trace; for the proton with C g5 (a real matrix) every weight
    is real, and each list has the normalisation of a projector (sum of the
    absolute weights equal for P+ and P-)."""
    tabs = {n: dict(zip(map(tuple, t), w)) for _, dss in prods for n, t, w in dss}
    pp, pm = tabs["proton/Pp_Cg5_Cg5"], tabs["proton/Pm_Cg5_Cg5"]
    assert all(abs(complex(v).imag) < 1e-7 for d in (pp, pm) for v in d.values())
    assert np.isclose(sum(abs(v) for v in pp.values()), sum(abs(v) for v in pm.values()))
    assert not set(pp) & set(pm)  # P+ and P- select different spin rows of the third quark
