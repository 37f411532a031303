/* Tile count of a BLAS matrix dimension (include/xkrt/memory/access/blas/matrix.h of the reference). */
#ifndef XKRT_B200_BLAS_MATRIX_H
#define XKRT_B200_BLAS_MATRIX_H
#define NUM_OF_TILES(N, TILE_SIZE) (((N) + (TILE_SIZE) - 1) / (TILE_SIZE))
#endif
