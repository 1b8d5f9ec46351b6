"""Result files in the reference's pickle formats (names, array shapes, row
schema) and the interval-march resume state read back from window files."""
import pickle

import numpy as np

from inching_b200 import results


def test_save_modes_formats(tmp_path):
    ev = np.array([0.1, 0.2, 0.35])
    modes = np.random.default_rng(0).standard_normal((3, 7, 3))
    paths = results.save_modes(str(tmp_path), "TRLMHD", "1abc", "Linux", "NVIDIA B200", ev, modes, pdbfn="x.pdb",
                               runtime=1.5, peak_mem_mib=10.0, residuals=[1e-9, 2e-9, 3e-9])
    names = sorted(p.split("/")[-1] for p in paths)
    assert names == ["Eigval_InchingTRLMHD_1abc_Linux_NVIDIAB200.pkl", "Eigvec_InchingTRLMHD_1abc_Linux_NVIDIAB200.pkl",
                     "PerformanceList_InchingTRLMHD_1abc_Linux_NVIDIAB200.pkl"]
    with open(paths[0], "rb") as fn:
        assert np.array_equal(pickle.load(fn), ev)
    with open(paths[1], "rb") as fn:
        assert pickle.load(fn).shape == (3, 7, 3)
    with open(paths[2], "rb") as fn:
        rows = pickle.load(fn)
    assert len(rows) == 3 and len(rows[0]) == 11
    assert rows[2][:3] == ["Inching (TRLMHD Linux NVIDIA B200)", "x.pdb", 7]
    assert rows[2][8:] == [2, 3e-9, 0.35]
    assert results.result_exists(str(tmp_path), "TRLMHD", "1abc", "Linux", "NVIDIA B200")


def test_window_files_and_resume_state(tmp_path):
    f = str(tmp_path)
    assert results.load_progress(f, "s", "Linux", "dev", 100) is None
    results.save_window(f, "s", "Linux", "dev", 0, np.array([0.5, 0.7, 0.9]), [1e-9] * 3, 120, runtime=2.0)
    results.save_window(f, "s", "Linux", "dev", 3, np.array([0.9, 1.2, 1.6, 2.0]), [1e-9] * 4, 300, runtime=5.0)
    st = results.load_progress(f, "s", "Linux", "dev", 100, plus_i=1.0)
    assert st["next_offset"] == 7 and st["remaining"] == 93
    assert abs(st["left_bound"] - (3.0 - 1e-10)) < 1e-12
    assert abs(st["interval_guess"] - 1.1) < 1e-12 and st["cumulative_runtime"] == 5.0
    with open(tmp_path / "PerformanceList_InchingManyCTRLM_s_Linux_dev_3.pkl", "rb") as fn:
        rows = pickle.load(fn)
    assert rows[0][0].startswith("Inching (CTRLM Interior") and rows[0][-2:] == [300, 3]
