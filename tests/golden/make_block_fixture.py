"""Writes tests/golden/block_matrix.json from the reference's block-matrix
known-answer test (raptor/core/tests/test_block_matrix.cpp, TEST
BlockMatrixTest): the 3 x 3 block matrix of 2 x 2 blocks it builds twice,
as blocks (BCOOMatrix::add_value per block, converted to BSR) and as scalar
entries (COOMatrix::add_value per entry, converted to CSR).  The test asserts
that both give the same products and the same CSR entries, so the fixture
holds both inputs; the checks are in tests/test_bsr.py.

    RAPTOR_REFERENCE_ROOT=<checkout> python tests/golden/make_block_fixture.py
"""
import json
import os
import re

REF = os.environ.get("RAPTOR_REFERENCE_ROOT", "/root/reference")
SRC = os.path.join(REF, "raptor", "core", "tests", "test_block_matrix.cpp")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "block_matrix.json")


def main():
    text = open(SRC).read()
    body = text[text.index("TEST(BlockMatrixTest"):]
    ints = {m.group(1): int(m.group(2))
            for m in re.finditer(r"int\s+(\w+)\s*=\s*(\d+)\s*;", body)}
    lists = {}
    for m in re.finditer(r"aligned_vector<(int|double)>\s+(\w+)\s*=\s*\{([^}]*)\}", body):
        kind, name, items = m.groups()
        conv = int if kind == "int" else float
        lists[name] = [conv(t) for t in items.replace("\n", " ").split(",") if t.strip()]
    fixture = {
        "source": "raptor/core/tests/test_block_matrix.cpp",
        "block_num_rows": ints["block_num_rows"],
        "block_num_cols": ints["block_num_cols"],
        "block_row_size": ints["block_row_size"],
        "block_col_size": ints["block_col_size"],
        "block_rows": lists["block_rows"],
        "block_cols": lists["block_cols"],
        # block k's values: vals[k * block_size : (k + 1) * block_size]
        "vals": lists["vals"],
        # the same matrix entry by entry (COOMatrix::add_value drops |v| <= 1e-16)
        "rows": lists["rows"],
        "cols": lists["cols"],
    }
    assert len(fixture["block_rows"]) == ints["block_nnz"]
    assert len(fixture["vals"]) == ints["block_nnz"] * ints["block_size"] == len(fixture["rows"])
    with open(OUT, "w") as f:
        json.dump(fixture, f, indent=1)
        f.write("\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
