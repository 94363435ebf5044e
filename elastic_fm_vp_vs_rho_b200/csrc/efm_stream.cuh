// Geometry of the plane-streaming kernels (efm_stream.cu).
#pragma once

#define EFM_STX 64          // tile width along x (cells) = threads per z-row
#define EFM_STZ 8           // tile rows along z; each thread computes rows r and r + 4
#define EFM_STHREADS 256
#define EFM_SR 4            // ring depth: planes j-1, j, j+1 resident, j+2 in flight
#define EFM_HX 72           // halo box width: x0-4 .. x0+67 (TMA x start stays 16-byte aligned)
#define EFM_HX_OFF 4
#define EFM_HZ 10           // halo box rows: z0-1 .. z0+8
#define EFM_HALO_TX (EFM_HX * EFM_HZ * 4)        // bytes one halo tile transfers (2880)
#define EFM_HALO_BYTES 2944                      // ... padded to a 128-byte multiple
#define EFM_CENTER_TX (EFM_STX * EFM_STZ * 4)    // bytes one cell tile transfers (2048)
#define EFM_CENTER_BYTES EFM_CENTER_TX
#define EFM_MAX_YCHUNK 64   // planes per block (bit mask of receiver planes is 64 bits)
