"""kmertreecounter_b200 -- B200-native exact canonical k-mer counter.

Drop-in for the counting path of ScorchShana/KmerTreeCounter: FASTQ in,
tmp/low.bin and tmp/root_{id}.bin out, in the reference's formats.  The
compute path is libkmertree_b200.so (sm_100a kernels behind the C ABI in
include/kmer_count.h); this package is its Python binding.
"""
from ._native import (  # noqa: F401
    ABI_SYMBOLS, KC_ERR_DEVICE, KC_ERR_INVALID, KC_ERR_IO, KC_ERR_NOMEM, KC_ERR_OVERFLOW, KC_ERR_STATE, KC_OK,
    KC_SINK_LOW, KC_SINK_ROOT, KC_SIZING_LEARNED, KC_SIZING_SAMPLED, Counter, KcConfig, KcError, KcStats, count_fastq, default_config,
    host_alloc, host_free, last_error, lib, measure_peaks, packed_bytes, record_bytes, record_dtype, stage0_file,
    stage0_rule, post_process_dir,
)
