"""CPU-side checks of the C ABI: the library loads and exports every symbol
that include/emb200.h declares, and host-only entry points (recipe, schedule)
agree with the oracle. No GPU is needed."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "emb200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|double|const char\*)\s+(emb200_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    syms = header_symbols()
    for s in ["emb200_create", "emb200_set_centroids", "emb200_set_bias", "emb200_assign_f32", "emb200_assign_i8",
              "emb200_assign_u8", "emb200_train", "emb200_load_rows", "emb200_assign_resident"]:
        assert s in syms


def test_library_exports_every_symbol(emb):
    L = emb.lib()
    for s in header_symbols():
        assert hasattr(L, s), s
        assert ctypes.cast(getattr(L, s), ctypes.c_void_p).value


def test_create_without_gpu_fails_cleanly(emb):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(emb.EngineError):
        emb.B200Assigner()


def test_recipe_matches_oracle(emb, orc):
    for (n, d, k, ne) in [(200_000, 96, 1024, 5.0), (1_000_000, 8, 100, 2.5), (4000, 4, 8, 5.0), (1000, 2, 10, 5.0),
                          (1_000_000, 128, 16384, 5.0), (2_000_000, 512, 4096, 5.0), (10_000_000, 96, 65536, 5.0),
                          (20_000, 64, 78, 5.0), (4_000_000, 8, 256, 5.0), (123, 7, 5, 0.3)]:
        a = emb.resolve_recipe(n, d, k, emb.Config(nepochs=ne))
        b = orc.resolve_recipe(n, d, k, orc.make_config(nepochs=ne))
        assert a.batch_size == b["batch_size"] and a.epoch_rows == b["epoch_rows"]
        assert a.alpha0 == b["alpha0"] and a.total_steps == b["total_steps"]
        assert a.unused_threshold == b["unused_threshold"]
    # src/lib.rs:526-540 goldens through the engine's own host code.
    r = emb.resolve_recipe(200_000, 96, 1024)
    assert r.batch_size == 16384 and abs(r.alpha0 - 0.728183) < 1e-5
    assert emb.scheduled_alpha(0.5, 100, 100) == pytest.approx(0.05, abs=1e-12)


def test_balance_stats_matches_oracle(emb, orc):
    import numpy as np

    lab = np.random.default_rng(0).integers(0, 50, 10_000).astype(np.uint32)
    a = emb.balance_stats(lab, 64)
    b = orc.balance_stats(lab, 64)
    assert a[0] == pytest.approx(b[0]) and a[1] == pytest.approx(b[1]) and a[2] == b[2]
