// Host-side interface of the single-pass index kernel (index_kernel.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace gpj {

constexpr int64_t kIndexTileBytes = 16384;  // exact kernel
// The line-parallel kernel owns 14 KiB per tile and reads 2 KiB past it, so
// that a tile and its look-ahead are one 64-byte word per index thread.
constexpr int64_t kLineTileBytes = 14336;
// The standalone index kernel owns 30 KiB per tile and reads 2 KiB past it:
// four consecutive 64-byte words per thread of a 128-thread CTA.
constexpr int64_t kStandaloneTileBytes = 30720;

// The file a tile of the standalone index kernel belongs to.  A build over
// one file uses IndexParams' own fields; a batch passes one entry per file,
// tiles numbered consecutively over the files (tile_begin = the file's first
// tile), positions and outputs relative to the file.
struct TileFile {
    const uint8_t* file;
    int64_t n;
    int64_t avail;            // bytes [0, avail) readable
    uint64_t* string_index;
    uint64_t* leveled;        // num_levels * level_size words
    int64_t level_size;
    uint64_t* newline_bits;
    unsigned long long* status;  // [0] line count, [1] error bits
    int64_t tile_begin;
    uint64_t* colon;          // optional: ':' outside strings (level_size words)
};

struct IndexParams {
    const uint8_t* file;
    int64_t n;
    int64_t ntiles;
    uint64_t* string_index;  // ceil(n/64)
    uint64_t* leveled;       // num_levels * level_size
    int64_t level_size;      // ceil(n/64)
    int num_levels;
    int64_t* newlines;  // newline_cap entries
    int64_t newline_cap;
    unsigned long long* tile_state;  // 3 * ntiles words, tagged with `epoch`
    unsigned int* tile_counter;      // zeroed before the launch; the exact and standalone kernels claim tiles from it
    unsigned long long* status;      // [0] line count, [1] error bits (zeroed before)
    uint32_t epoch;                  // 1..65535
    int materialize;                 // write string_index / leveled / newlines
    // Line-parallel kernel only: this launch indexes tiles [tile_begin,
    // tile_end) (earlier tiles were indexed by earlier launches of the same
    // build, with the same epoch), and only bytes [0, avail) of the file may
    // be read (the rest may still be on its way from the host; avail is n or
    // a multiple of 64 at or past the end of the last tile's following
    // tile).  A line that runs past `avail` is flagged kErrLongLine.
    int64_t tile_begin;
    int64_t tile_end;
    int64_t avail;
    // Standalone index kernel only: the '\n' bitmap (ceil(n/64) words) and
    // the newline count of every tile, in place of the newline index.
    uint64_t* newline_bits;
    int32_t* tile_newlines;
    // Standalone kernel, optional: the ':' bytes outside strings
    // (ceil(n/64) words), which lets find_value's key searches skip the ','
    // candidates.
    uint64_t* colon;
    // Standalone kernel over a batch of files (batch_files > 0): tiles
    // [tile_begin, tile_end) of the whole batch, file table `batch`
    // (ascending tile_begin); status then reports errors that concern no
    // single file (wait timeouts).
    const TileFile* batch;
    int batch_files;
    // Longest run past its tile a CTA follows to finish a line before it
    // flags kErrLongLine (0: the kernels' default, 64 KiB).
    int64_t max_extension;

    // Queries evaluated in the same pass (line-parallel kernel only; 0 = none).
    int num_queries;
    const uint8_t* bytecode;  // all queries back to back
    int bytecode_bytes;       // total length of `bytecode`
    const int32_t* offsets;   // start of query q in `bytecode`
    int slots;
    int64_t* out;       // [num_queries][out_lines][slots][2]
    int64_t out_lines;  // line capacity of `out` (its query stride)
};

// Exact kernel: carries string state, level and newline count across tiles
// by decoupled look-back; correct for any input.
cudaError_t launch_index_kernel(const IndexParams& p, int grid, cudaStream_t stream);
int index_kernel_max_ctas_per_sm(int num_levels);

// Line-parallel kernel for NDJSON: every line starts outside strings at
// level -1; flags kErrIrregular / kErrLongLine when that does not hold and
// the exact kernel must be used.  tile_state needs 2 * ntiles words.
cudaError_t launch_line_index_kernel(const IndexParams& p, int grid, cudaStream_t stream);
int line_index_max_ctas_per_sm(int num_levels);

// Standalone form of the line-parallel kernel for index builds without
// in-kernel queries: the index warps alone (up to five CTAs per SM), no tile
// depending on another; writes string index and leveled bitmaps, and
// newline_bits + tile_newlines instead of the newline index (same error
// flags).  launch_newline_index then builds the newline index.
cudaError_t launch_tile_index_kernel(const IndexParams& p, int grid, cudaStream_t stream);
int tile_index_max_ctas_per_sm(int num_levels);

// Newline index from newline_bits and tile_newlines (tiles of
// kStandaloneTileBytes): offsets of the tile counts within blocks of 1024 tiles
// and the block sums into `offsets` (newline_offsets_words(ntiles)
// entries), then every tile's '\n' positions; writes status[0] =
// newlines + 1 and at most newline_cap entries.  Two launches, one stream.
cudaError_t launch_newline_index(const IndexParams& p, int64_t* offsets, int grid, cudaStream_t stream);
// The same for tiles [t0, t1) only, once every earlier tile's newline index
// is written (t0 and, unless t1 = ntiles, t1 multiples of 1024); the number
// of lines whose both ends are then known goes to device memory
// `lines_done` (the newlines up to tile t1 - 1, + 1 for the last line when
// t1 = ntiles).
cudaError_t launch_newline_index_range(const IndexParams& p, int64_t* offsets, int64_t t0, int64_t t1,
                                       int64_t* lines_done, int grid, cudaStream_t stream);
inline int64_t newline_offsets_words(int64_t ntiles) { return ntiles + (ntiles + 1023) / 1024; }

// Where the newline index of one file of a batch goes.
struct LineFile {
    const uint64_t* newline_bits;
    int64_t words;               // ceil(n / 64)
    int64_t* newlines;
    int64_t cap;                 // entries `newlines` holds
    unsigned long long* status;  // [0] receives the line count
    int64_t tile_begin;          // the file's first tile in the batch
    int64_t ntiles;
};

// Newline indexes of a batch (tile_newlines of all its tiles, ascending
// tile_begin in `files`, a device array of nfiles entries).
cudaError_t launch_newline_index_batch(const int32_t* tile_newlines, int64_t total_tiles, const LineFile* files,
                                       int nfiles, int64_t* offsets, int grid, cudaStream_t stream);

}  // namespace gpj
