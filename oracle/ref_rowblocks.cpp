// C entry around the reference's own ComputeRowBlocks
// (src/library/internal/data-types/csr-meta.hpp:93-269), compiled straight
// from the reference sources by oracle/Makefile into oracle/_ref/. Test
// infrastructure only: it produces the golden row-block words the oracle and
// the library are checked against.
#include "internal/data-types/csr-meta.hpp"

extern "C" {

// Size-only run (ComputeRowBlocksSize).
unsigned int ref_row_blocks_size(const unsigned int* rp, unsigned int n) {
    return static_cast<unsigned int>(ComputeRowBlocksSize(rp, n, BLKSIZE, BLOCK_MULTIPLIER, ROWS_FOR_VECTOR));
}

// Fills `words` (capacity from ref_row_blocks_size / 2 + 1) and returns the
// rowBlockSize the reference stores in its meta.
unsigned int ref_row_blocks(const unsigned int* rp, unsigned int n, unsigned long long* words,
                            unsigned int capacity_words) {
    clsparseIdx_t size = capacity_words * 2;
    ComputeRowBlocks(reinterpret_cast<cl_ulong*>(words), size, rp, n, BLKSIZE, BLOCK_MULTIPLIER,
                     ROWS_FOR_VECTOR, true);
    return size;
}

// Same with a chosen row-block shape (blkSize, blkMultiplier, rows_for_vector
// are parameters of the reference's ComputeRowBlocks; the library's
// clsparseB200CsrMetaCreateTuned must reproduce these words).
unsigned int ref_row_blocks_shape_size(const unsigned int* rp, unsigned int n, unsigned int blk, unsigned int mult,
                                       unsigned int rfv) {
    return static_cast<unsigned int>(ComputeRowBlocksSize(rp, n, blk, mult, rfv));
}

unsigned int ref_row_blocks_shape(const unsigned int* rp, unsigned int n, unsigned int blk, unsigned int mult,
                                  unsigned int rfv, unsigned long long* words, unsigned int capacity_words) {
    clsparseIdx_t size = capacity_words * 2;
    ComputeRowBlocks(reinterpret_cast<cl_ulong*>(words), size, rp, n, blk, mult, rfv, true);
    return size;
}

}
