"""Result files (qmcrt_write_flux_csv / qmcrt_write_intercept_ratio) against
the text the reference's own ImageSaver::savetxt (image_save.cpp:5-48)
wrote for the same seeded map (tests/golden/ref_host_vectors.npz, made by
tests/golden/gen_ref_vectors.py): byte for byte, appending twice."""
import os

import numpy as np
import pytest

from onemirror_b200 import capi
from onemirror_b200.scene import write_flux_csv, write_intercept_ratio

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_host_vectors.npz"))


@pytest.mark.parametrize("precision,key", [(2, "save_flux_p2"), (4, "save_flux_p4")])
def test_flux_file_equals_reference_bytes(tmp_path, precision, key):
    path = tmp_path / "flux.txt"
    write_flux_csv(path, G["save_map"], precision=precision)
    write_flux_csv(path, G["save_map"], precision=precision)
    assert path.read_bytes() == G[key].tobytes()


def test_intercept_file_equals_reference_bytes(tmp_path):
    path = tmp_path / "ratio.txt"
    total = float(G["save_total"])
    r = write_intercept_ratio(path, G["save_map"], total)
    write_intercept_ratio(path, G["save_map"], total)
    assert path.read_bytes() == G["save_ratio"].tobytes()
    # the ratio is the float32 sum in the file's order (last row first)
    m = G["save_map"]
    acc = np.float32(0)
    for row in m[::-1]:
        for v in row:
            if not float(v) < 1e-6:
                acc = np.float32(acc + v)
    assert r == float(np.float32(acc / np.float32(total)))
    assert write_intercept_ratio(None, m, total) == r


def test_overwrite_and_errors(tmp_path):
    path = tmp_path / "flux.txt"
    write_flux_csv(path, G["save_map"], precision=2)
    write_flux_csv(path, G["save_map"], precision=2, append=False)
    assert path.read_bytes() == G["save_flux_p2"].tobytes()[: len(G["save_flux_p2"]) // 2]
    with pytest.raises(capi.QmcrtError):
        write_flux_csv(tmp_path / "no_such_dir" / "f.txt", G["save_map"])
    with pytest.raises(capi.QmcrtError):
        write_flux_csv(path, G["save_map"], precision=-1)
    with pytest.raises(ValueError):
        write_flux_csv(path, G["save_map"].ravel())
