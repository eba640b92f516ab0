"""cohsearch -- B200 engine for CoherentSearch.jl's coherent search hot path.

The public names mirror the Julia API (src/CoherentSearch.jl:17-51); the hot
loop runs in ``libcohsearch_cuda.so`` (sm_100a) through its C ABI.
"""
from ._lib import CohSearchError, LIB_PATH, load as load_library
from .fileio import FFTFile, SimpleInf, freqs, write_fft
from .metricstats import (BlockMetricStats, MetricHistogram, MetricNorm, MetricStats, build_metricnorm,
                          hist_quantile, metricstats_summary, metricstats_windows)
from .search import (Candidate, Engine, SearchCache, SearchParams, block_metrics, boxcar_widths, candidate_profile,
                     chunk_metrics, measure_ducy, rotate_to_peak,
                     decimation_set, ladder_boxcar_widths, proftype, remove_duplicates,
                     remove_harmonics, search, search_batch, search_block, write_candidates, output_path,
                     search_files)

__all__ = [
    "CohSearchError", "LIB_PATH", "load_library", "FFTFile", "SimpleInf", "freqs", "write_fft",
    "Candidate", "Engine", "SearchCache", "SearchParams", "boxcar_widths", "chunk_metrics",
    "decimation_set", "ladder_boxcar_widths", "proftype", "remove_duplicates", "remove_harmonics",
    "search", "write_candidates", "BlockMetricStats", "MetricHistogram", "MetricNorm", "MetricStats",
    "build_metricnorm", "hist_quantile", "metricstats_summary", "metricstats_windows", "block_metrics",
    "search_block", "search_batch", "candidate_profile", "measure_ducy", "rotate_to_peak", "output_path",
    "search_files",
]
