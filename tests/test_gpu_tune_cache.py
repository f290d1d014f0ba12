"""Measured MSM window widths saved and loaded across contexts (nkr_b200_tune_save /
nkr_b200_tune_load): a loaded context reports the saved width and time without
measuring again; files of another device or of another format are refused."""
import pytest

import nkr_b200 as nk

pytestmark = pytest.mark.gpu


def test_tune_cache_round_trip(tmp_path):
    path = tmp_path / "tune.txt"
    a = nk.Context(0)
    c, ms = a.tune_msm(1 << 14)
    a.tune_save(path)
    a.close()
    text = path.read_text()
    assert text.startswith("nkr-b200-tune 1\n") and "msm 14 %d " % c in text
    b = nk.Context(0)
    assert b.tune_load(path) >= 1
    c2, ms2 = b.tune_msm(1 << 14)
    assert c2 == c and abs(ms2 - ms) < 1e-3     # the loaded entry, not a new measurement
    b.close()


def test_tune_cache_refuses_foreign_files(tmp_path):
    ctx = nk.Context(0)
    other = tmp_path / "other.txt"
    other.write_text("nkr-b200-tune 1\ndevice Some Other GPU\nsms 7\nmsm 14 12 1.0\n")
    with pytest.raises(nk.B200Error):
        ctx.tune_load(other)
    junk = tmp_path / "junk.txt"
    junk.write_text("not a tuning file\n")
    with pytest.raises(nk.B200Error):
        ctx.tune_load(junk)
    ctx.close()
