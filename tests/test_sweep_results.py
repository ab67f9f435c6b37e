"""The batched sweep's result tables (results.csv, layers.csv, checksums.json):
their layout, on made-up tables (no GPU)."""
import csv
import hashlib
import json

from multigpubfs_b200.batch import write_sweep_results


def test_layout_and_checksums(tmp_path):
    tables = [[1, 3, 4], [], [1, 2, 2, 1]]
    seconds = [[0.0, 1e-3, 2e-3], [], [0.0, 1e-4, 2e-4, 3e-4]]
    sums = write_sweep_results(tmp_path, ["a", "b", "c"], [3, 5, 4], tables, seconds)
    with open(tmp_path / "results.csv", newline="") as f:
        rows = list(csv.DictReader(f))
    assert [r["status"] for r in rows] == ["COMPLETE", "INCOMPLETE", "COMPLETE"]
    assert rows[0]["eccentricity"] == "2" and rows[0]["visited"] == "8" and rows[1]["eccentricity"] == ""
    assert abs(float(rows[2]["bfs_seconds"]) - 6e-4) < 1e-12
    with open(tmp_path / "layers.csv", newline="") as f:
        layers = list(csv.DictReader(f))
    assert [(r["instance"], r["depth"], r["count"], r["cumulative"]) for r in layers] == [
        ("0", "0", "1", "1"), ("0", "1", "3", "4"), ("0", "2", "4", "8"),
        ("2", "0", "1", "1"), ("2", "1", "2", "3"), ("2", "2", "2", "5"), ("2", "3", "1", "6")]
    assert layers[0]["seconds"] == "" and float(layers[1]["seconds"]) == 1e-3
    disk = json.loads((tmp_path / "checksums.json").read_text())
    assert disk == sums
    for name, digest in sums.items():
        assert hashlib.sha256((tmp_path / name).read_bytes()).hexdigest() == digest
