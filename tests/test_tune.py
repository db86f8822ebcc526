"""Autotuner cache: lookup order (user cache, then the packaged B200 table) and the
JSON round trip. No GPU: the device name is passed explicitly."""
import json

from pfc_models_b200 import _lib, tune


def test_packaged_table_is_used_without_a_user_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("PFC_TUNE_CACHE", str(tmp_path / "none.json"))
    table = json.load(open(tune.PACKAGED))
    assert table, "the packaged table is empty"
    key = "NVIDIA B200|2048x2048|fp32|std"
    assert key in table
    v = tune.lookup(2048, 2048, _lib.FP32_MIXED, _lib.MODEL_STD, device_name="NVIDIA B200")
    assert v == {k: int(table[key].get(k) or 0) for k in tune.VARIANT_KEYS}
    for k, e in table.items():
        # 0: the plan's own choice (a side with an odd factor holds a fixed number per thread)
        assert e["ee_row"] in (0, 8, 16, 32) and e["ee_col"] in (0, 8, 16, 32) and 1 <= e["row_tile"] <= 16
        assert e.get("col_cta", 0) in (0, 1, 2, 4) and e.get("pdl", 0) in (0, 1, 2)
        assert e.get("packed") in (None, 0, 1, 2, 3) and e.get("tma") in (None, 0, 1)
        _, grid, prec, model = k.split("|")[:4]
        nx, ny = (int(x) for x in grid.split("x"))
        assert prec in ("fp32", "fp64") and model in ("std", "log"), k
        if prec == "fp64":
            # 16 complex doubles per thread at most; the two-lane kernels are FP32 only
            assert e["ee_row"] <= 16 and e["ee_col"] <= 16 and not e.get("packed") and not e.get("tma"), k
        assert e["ee_row"] <= nx // 2 and e["ee_col"] <= ny, k
        # every entry encodes into the plan's flag bits
        _lib.flag_variant(**{v: int(e.get(v) or 0) for v in tune.VARIANT_KEYS})
    # batch-measured entries are preferred for batches and fall back to the single-plan ones
    bkey = "NVIDIA B200|512x512|fp32|std|batch"
    assert bkey in table
    vb = tune.lookup(512, 512, _lib.FP32_MIXED, _lib.MODEL_STD, device_name="NVIDIA B200", batched=True)
    assert vb == {k: int(table[bkey].get(k) or 0) for k in tune.VARIANT_KEYS}
    v2 = tune.lookup(2048, 2048, _lib.FP32_MIXED, _lib.MODEL_STD, device_name="NVIDIA B200", batched=True)
    assert v2 == v
    assert tune.lookup(2048, 2048, _lib.FP32_MIXED, _lib.MODEL_STD, device_name="other GPU") is None


def test_user_cache_overrides_and_round_trips(tmp_path, monkeypatch):
    path = tmp_path / "sub" / "tune.json"
    monkeypatch.setenv("PFC_TUNE_CACHE", str(path))
    key = tune._key("NVIDIA B200", 2048, 2048, _lib.FP32_MIXED, _lib.MODEL_STD)
    tune._store(str(path), key, {"ee_row": 16, "ee_col": 32, "row_tile": 2, "row_us": 1.0, "col_us": 2.0})
    tune._memo.clear()
    assert json.load(open(path))[key]["ee_col"] == 32
    assert tune.lookup(2048, 2048, _lib.FP32_MIXED, _lib.MODEL_STD, device_name="NVIDIA B200") == \
        {"ee_row": 16, "ee_col": 32, "row_tile": 2, "col_cta": 0, "pdl": 0, "packed": 0, "tma": 0, "generic": 0}
    # entries of the second stage carry the column CTA width and the launch mode
    tune._store(str(path), key, {"ee_row": 16, "ee_col": 16, "row_tile": 4, "col_cta": 1, "pdl": 1})
    tune._memo.clear()
    assert tune.lookup(2048, 2048, _lib.FP32_MIXED, _lib.MODEL_STD, device_name="NVIDIA B200") == \
        {"ee_row": 16, "ee_col": 16, "row_tile": 4, "col_cta": 1, "pdl": 1, "packed": 0, "tma": 0, "generic": 0}
    tune._memo.clear()


def test_flag_encoding_matches_header():
    import re
    from tests.conftest import ROOT
    import os
    src = open(os.path.join(ROOT, "include", "pfc_b200.h")).read()
    shifts = dict(re.findall(r"#define PFC_FLAG_(ROW_EE|COL_EE|ROW_TILE)\(\w\) \(\(int32_t\)\(\w\) << (\d+)\)", src))
    assert shifts == {"ROW_EE": "8", "COL_EE": "16", "ROW_TILE": "24"}
    assert _lib.flag_variant(16, 32, 4) == (16 << 8) | (32 << 16) | (4 << 24)
    assert re.search(r"#define PFC_FLAG_PDL 4\b", src)
    # packed kernels: both passes by flag, one pass by the EE bit; TMA staging by flag
    assert re.search(r"#define PFC_FLAG_PACKED 16\b", src) and re.search(r"#define PFC_EE_PACKED 0x80\b", src)
    assert re.search(r"#define PFC_FLAG_TMA 64\b", src) and re.search(r"#define PFC_FLAG_EXTV 32\b", src)
    assert _lib.flag_variant(16, 32, 4, packed=1) & _lib.FLAG_PACKED
    assert (_lib.flag_variant(16, 32, 4, packed=2) >> 8) & 0xff == 16 | _lib.EE_PACKED
    assert (_lib.flag_variant(16, 16, 4, packed=3) >> 16) & 0xff == 16 | _lib.EE_PACKED
    assert _lib.flag_variant(16, 32, 8, packed=2, tma=1) & _lib.FLAG_TMA
    assert re.search(r"#define PFC_FLAG_COL_CTA\(c\) .*<< 29\)", src)
    # columns per CTA 1, 2, 4 -> field values 1, 2, 3 in bits 29-30
    assert [_lib.flag_variant(col_cta=c) >> 29 for c in (0, 1, 2, 4)] == [0, 1, 2, 3]
    assert _lib.flag_variant(pdl=1) == _lib.FLAG_PDL
    assert _lib.flag_variant(pdl=2) == _lib.FLAG_PDL_COL
    assert re.search(r"#define PFC_FLAG_PDL_COL 128", src)


def test_refine_keeps_defaults_unless_clearly_faster(monkeypatch):
    """Second stage: (columns per CTA, programmatic launch of both kernels or the column
    kernel only) is taken from whole-step
    timings only when at least 1 % faster than the defaults; choices whose launch equals
    one timed already (same column-kernel threads) are not timed again. The timings are
    faked, so this runs without a GPU."""
    calls = []

    def fake(times, threads):
        def _time_blocks(nx, ny, precision, model, variant, batch, steps=320, skip=None):
            key = (variant["col_cta"], variant["pdl"])
            th = threads[variant["col_cta"]]
            if skip is not None and skip(th):
                return None, th
            calls.append(key)
            return times[key], th
        return _time_blocks

    base = {"ee_row": 32, "ee_col": 16, "row_tile": 8}
    # 256 threads by default (2 columns of 128); 4 columns clamp to the same launch
    threads = {0: 256, 1: 128, 2: 256, 4: 256}
    times = {(0, 0): 40.0, (0, 1): 39.8, (0, 2): 39.9, (1, 0): 45.0, (1, 1): 47.0, (1, 2): 46.0}
    monkeypatch.setattr(tune, "_time_blocks", fake(times, threads))
    r = tune.refine(2048, 2048, "fp32", "std", base)
    assert (r["col_cta"], r["pdl"]) == (0, 0)            # 0.5 % faster is not enough
    # 2 and 4 columns per CTA launch like the default here: skipped, not timed
    assert calls == [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2)]
    assert set(r["refine_us"]) == {"0/0", "0/1", "0/2", "1/0", "1/1", "1/2"}
    calls.clear()
    times = {(0, 0): 12.0, (0, 1): 11.5, (0, 2): 11.6, (1, 0): 9.4, (1, 1): 8.6, (1, 2): 8.9}
    monkeypatch.setattr(tune, "_time_blocks", fake(times, {0: 256, 1: 128, 2: 256, 4: 256}))
    r = tune.refine(128, 128, "fp32", "std", base)
    assert (r["col_cta"], r["pdl"]) == (1, 1)
    # a grid the fast kernels do not cover keeps the defaults
    monkeypatch.setattr(tune, "_time_blocks", lambda *a, **k: (None, None))
    assert tune.refine(96, 96, "fp32", "std", base) == {"col_cta": 0, "pdl": 0}
