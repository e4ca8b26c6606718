"""The FlyWire v783 file loader (CPU): a tiny data directory in the three files' formats; the
biological sign corrections against the reference's own outputs."""

import numpy as np
import pandas as pd

from flyzero_b200 import connectome as cx


def test_load_flywire_files(tmp_path):
    ids = np.array([720575940600000001, 720575940600000002, 720575940600000003, 720575940600000004], np.int64)
    pd.DataFrame({"Completed": [True] * 4}, index=pd.Index(ids, name="Unnamed: 0")).to_csv(tmp_path / "Completeness_783.csv")
    con = pd.DataFrame({"Presynaptic_Index": [0, 0, 1, 3, 0], "Postsynaptic_Index": [1, 2, 2, 0, 1],
                        "Excitatory x Connectivity": [5, -2, 7, 3, 1]})
    con.to_parquet(tmp_path / "Connectivity_783.parquet")
    ann = pd.DataFrame({"root_id": ids[[2, 0, 1, 3]], "root_630": ids[[2, 0, 1, 3]] - 5,
                        "cell_type": ["DNg02_a", "DNa02", "DNa02", "MDN"], "hemibrain_type": [None, None, None, "MDN_x"],
                        "side": ["left", "left", "right", "left"], "super_class": ["descending"] * 4})
    ann.to_csv(tmp_path / "neuron_annotations.tsv", sep="\t", index=False)
    c = cx.load_flywire(tmp_path)
    assert c.n == 4 and c.weights.dtype == np.float32
    dense = c.weights.toarray()
    assert dense[0, 1] == 6 and dense[0, 2] == -2 and dense[1, 2] == 7 and dense[3, 0] == 3   # duplicates added
    assert list(c.find("DNa02")) == [0, 1]
    assert list(c.find("dna02", "right")) == [1]
    assert list(c.find("DNg02*")) == [2]
    assert list(c.find("MDN_x")) == [3]                       # hemibrain type
    assert list(c.neurons["root_id"]) == list(ids)


def test_biology_corrections_match_reference(golden):
    """``corrected`` against the reference's own biology.corrected (tests/golden/biology.npz)."""
    import os
    import sys

    import scipy.sparse as sp

    from flyzero_b200.connectome import Connectome, corrected

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_biology_golden as G

    z = golden("biology.npz")
    n = len(z["nt"])
    w = sp.csr_matrix((z["w_data"], z["w_indices"], z["w_indptr"]), shape=(n, n))
    df = G.neurons(z["nt"].astype(str), z["cls"].astype(str))
    for name, fixes in G.FIXES.items():
        c = corrected(Connectome(w, df), fixes).weights.tocsr()
        c.sort_indices()
        np.testing.assert_array_equal(c.indptr, z[f"{name}_indptr"], err_msg=name)
        np.testing.assert_array_equal(c.indices, z[f"{name}_indices"], err_msg=name)
        np.testing.assert_array_equal(c.data, z[f"{name}_data"], err_msg=name)
