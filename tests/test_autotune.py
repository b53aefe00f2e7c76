"""The autotuner's table lookup (CPU, no GPU): nearest tuned dimension, ties
to the larger, built-in default without a table; the shipped table (when
present) holds a valid configuration for every entry."""
import hilbertjoin_b200.autotune as A


def test_lookup_nearest_and_default():
    t = {"entries": {"8": {"best": {"form": "tf32", "item_chunk": 8, "active_dims": 2, "ms": 1.0}},
                     "64": {"best": {"form": "fp16", "item_chunk": 32, "active_dims": 1, "ms": 3.0}}}}
    assert A.config_for(3, table=t) == {"form": "tf32", "item_chunk": 8, "active_dims": 2}
    assert A.config_for(36, table=t)["form"] == "fp16"  # tie between 8 and 64: the larger
    assert A.config_for(200, table=t)["item_chunk"] == 32
    assert A.config_for(10, table={"entries": {}}) == A.DEFAULT


def test_shipped_table_is_valid():
    t = A.load_table()
    if t is None:
        return
    for d, e in t["entries"].items():
        b = e["best"]
        assert b["form"] in A.FORMS and b["item_chunk"] in A.CHUNKS and b["active_dims"] in A.ACTIVE
        assert e["count"] >= 0 and int(d) > 0
