// Supported FFT lengths and their four-step split N = N1 * N2 (N1 values per
// thread in step 1, N2 in step 2).  One list shared by the kernels and the host.
#pragma once

#define INQB_FFT_SIZES(X)                                                                     \
  X(12, 4, 3) X(16, 4, 4) X(18, 6, 3) X(20, 5, 4) X(24, 8, 3) X(30, 6, 5) X(32, 8, 4)        \
  X(36, 6, 6) X(40, 8, 5) X(48, 8, 6) X(60, 12, 5) X(64, 8, 8) X(72, 9, 8) X(80, 16, 5)     \
  X(96, 12, 8) X(128, 16, 8) X(144, 16, 9)
