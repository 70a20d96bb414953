/* FP64 CPU oracle of the cuVHS decode (TEST INFRASTRUCTURE ONLY).
 *
 * A plain C++ restatement of the reference decoder's algorithm, stage by stage
 * and with the reference's tiling (spp-stride tiles, 2048-sample overlap-save
 * trash zone, chunk restarts), used by the tests as the parity checker and by
 * bench.py as the host-core CPU baseline.  Nothing in the product links or
 * calls it.  Each function cites the reference file:line it follows.
 *
 * Parity pin: the oracle is checked against the reference's own outputs (CUDA
 * build compiled from the reference sources and run on a B200; fixtures under
 * tests/golden/ with the script that generated them).
 */
#ifndef CUVHS_ORACLE_H
#define CUVHS_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;

/* mhz: capture rate; batch_fields: the reference's chunk size in fields
 * (its VRAM-derived batch_size); threads: host threads (0 = all cores). */
oracle_ctx* oracle_create(double mhz, int batch_fields, int threads); /* NTSC */
/* system: 0 NTSC, 1 PAL (VideoFormat's two branches, video_format.cpp:23-104) */
oracle_ctx* oracle_create_system(double mhz, int batch_fields, int threads, int system);
/* output field geometry and line locations per field of the context's system */
int oracle_field_width(const oracle_ctx* c);
int oracle_field_height(const oracle_ctx* c);
int oracle_lines_per_frame(const oracle_ctx* c);
void oracle_destroy(oracle_ctx* c);

/* Decode a whole u8 capture held in memory.  Returns number of fields. */
int oracle_decode(oracle_ctx* c, const uint8_t* data, size_t n);

/* Results of the last decode. */
int oracle_num_fields(const oracle_ctx* c);
const uint16_t* oracle_luma(const oracle_ctx* c);    /* [fields][height][width] */
const uint16_t* oracle_chroma(const oracle_ctx* c);  /* [fields][height][width] */
/* The .tbc.json text the reference writer would produce (NUL-terminated). */
const char* oracle_json(const oracle_ctx* c);

/* Per-chunk intermediates (chunk index k). */
int oracle_num_chunks(const oracle_ctx* c);
/* meta: raw_offset, fields, spp, tiles, requested_fields, next_raw_offset */
void oracle_chunk_meta(const oracle_ctx* c, int k, long long meta[6]);
/* Copy an intermediate array of chunk k into dst (count elements); returns
 * the element count (call with dst = NULL to query).  Names: "vsync_candidates",
 * "field_offsets"(i64), "k2_pulse_count", "k2_pulse_starts", "k2_pulse_lengths",
 * "k2b_pulse_count", "k2b_pulse_starts", "k2b_pulse_lengths", "k2b_pulse_types",
 * "is_first", "do_count", "do_lines", "do_starts", "do_ends" (i32);
 * "linelocs_coarse", "linelocs", "demod", "demod05", "envelope",
 * "chroma_prefilt" (f64). */
long long oracle_chunk_array(const oracle_ctx* c, int k, const char* name, void* dst, long long cap);

/* Keep the per-chunk FP64 sample arrays (demod, demod05, envelope,
 * chroma_prefilt) of chunk 0 for inspection (memory heavy). */
void oracle_keep_signals(oracle_ctx* c, int keep);
/* Capture sample format (0 u8, 1 s16, 2 u16; oracle_decode's data then holds
 * 1 or 2 bytes per sample and n counts samples) and DC correction, as the
 * reference's --format and --dc-correct. */
void oracle_set_input(oracle_ctx* c, int format, int dc_correct);
/* The reference's K3 line locations in place of K2b, as its CUVHS_K2B_DISABLE
 * environment switch (which the oracle also honours). */
void oracle_set_single_pass(oracle_ctx* c, int on);

#ifdef __cplusplus
}
#endif
#endif
