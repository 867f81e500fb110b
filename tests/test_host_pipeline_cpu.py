"""CPU tests of HostPipeline's chunking rule: chunks of whole detectors that cover every detector
once, each a multiple of 32 samples (the plan's cache-line unit), about the requested size."""

import pytest

from gpu_mm_b200.host_pipeline import chunk_plan


@pytest.mark.parametrize("ndet,nt,chunk_dets", [(1024, 2 ** 18, None), (10, 1008, 3), (7, 1024, 2), (5, 4096, None),
                                                (96, 100, 5), (33, 96, 64), (1, 2 ** 20, None)])
def test_chunks_cover_detectors_in_cache_lines(ndet, nt, chunk_dets):
    cd, chunks = chunk_plan(ndet, nt, chunk_dets)
    assert chunks[0][0] == 0 and chunks[-1][1] == ndet
    assert all(a[1] == b[0] for a, b in zip(chunks, chunks[1:]))
    assert all(((d1 - d0) * nt) % 32 == 0 and d1 > d0 for d0, d1 in chunks)
    assert all(d1 - d0 == cd for d0, d1 in chunks[:-1])
    if chunk_dets is None:
        assert cd * nt <= max(1 << 24, nt * 32)


def test_default_chunk_size_for_the_bench_workload():
    cd, chunks = chunk_plan(1024, 2 ** 18)
    assert cd == 64 and len(chunks) == 16          # 2^24 samples per chunk


def test_bad_sizes_rejected():
    with pytest.raises(RuntimeError, match="multiple of 32"):
        chunk_plan(3, 7)
    with pytest.raises(RuntimeError, match="multiple of 32"):
        chunk_plan(0, 64)
