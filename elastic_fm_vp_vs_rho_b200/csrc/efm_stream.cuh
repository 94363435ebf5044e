// Geometry of the plane-streaming kernels (efm_stream.cu).
//
// A block owns a 64-wide (x) column of 4 * ROWS z-rows and marches along y; each of its 256
// threads computes ROWS cells per plane (rows r, r + 4, ...).  ROWS = 2 (64 x 8 tiles, two
// blocks per SM) and ROWS = 1 (64 x 4 tiles, three blocks per SM with a 4-deep ring, two
// with a 6-deep ring that keeps four planes in flight) are built.
#pragma once

#define EFM_STX 64          // tile width along x (cells) = threads per z-row
#define EFM_STZ 8           // tile rows along z of the two-row variant
#define EFM_STHREADS 256
#define EFM_SR 4            // default ring depth: planes j-1, j, j+1 resident, j+2 in flight
#define EFM_HX 72           // halo box width: x0-4 .. x0+67 (TMA x start stays 16-byte aligned)
#define EFM_HX_OFF 4
#define EFM_REC_TZ 4        // z granularity of the per-tile receiver map
#define EFM_MAX_YCHUNK 64   // planes per block (bit mask of receiver planes is 64 bits)

// Box and shared-memory sizes of the variant computing `rows` cells per thread.
__host__ __device__ constexpr int efm_st_tz(int rows) { return 4 * rows; }
__host__ __device__ constexpr int efm_st_hz(int rows) { return 4 * rows + 2; }  // z0-1 .. z0+tz
__host__ __device__ constexpr int efm_halo_tx(int rows) { return EFM_HX * efm_st_hz(rows) * 4; }
__host__ __device__ constexpr int efm_halo_bytes(int rows) {
    return (efm_halo_tx(rows) + 127) / 128 * 128;
}
__host__ __device__ constexpr int efm_center_bytes(int rows) { return EFM_STX * efm_st_tz(rows) * 4; }
__host__ __device__ constexpr int efm_stream_smem(int rows, int sr, int nh, int nc) {
    return sr * (nh * efm_halo_bytes(rows) + nc * efm_center_bytes(rows));
}
// resident blocks per SM the launch bounds promise: 2 for two rows or a 6-deep ring, else 3
__host__ __device__ constexpr int efm_stream_blocks(int rows, int sr) {
    return rows == 1 && sr == 4 ? 3 : 2;
}
