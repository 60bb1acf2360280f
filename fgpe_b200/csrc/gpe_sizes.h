// gpe_sizes.h -- grid lengths with compiled pass kernels, per family.  Each
// family is one translation unit per precision and field count
// (gpe_inst_<family>_<d|f><1|2>.cu); the long lengths sit in families of
// their own so that the units compile in similar times.
// GPE_DEV_SIZES (make GPE_DEV=1) keeps only the lengths the test suite uses,
// for quick kernel rebuilds during development.
#pragma once
// GPE_TUNED_*: the lengths of the benchmark configurations, which also carry
// the strided-pass variants the autotuner chooses from (gpe_tune.cu).
#ifdef GPE_DEV_SIZES
#define GPE_TUNED_p2(X) X(64)
#define GPE_TUNED_p2b(X) X(128)
#define GPE_TUNED_p3b(X) X(96)
#else
#define GPE_TUNED_p2(X) X(64)
#define GPE_TUNED_p2b(X) X(128) X(256) X(512)
#define GPE_TUNED_p3b(X) X(96) X(192) X(384)
#endif
#define GPE_TUNED_p3(X)
#define GPE_TUNED_p5(X)
#define GPE_TUNED_p5b(X)
#define GPE_TUNED_p9(X)
#define GPE_TUNED_p9b(X)
#ifdef GPE_DEV_SIZES
#define GPE_SIZES_p2(X) X(1) X(4) X(8) X(16) X(32) X(64)
#define GPE_SIZES_p2b(X) X(128)
#define GPE_SIZES_p3(X) X(6) X(12) X(24)
#define GPE_SIZES_p3b(X) X(96)
#define GPE_SIZES_p5(X) X(5) X(10) X(20) X(40) X(25)
#define GPE_SIZES_p5b(X)
#define GPE_SIZES_p9(X) X(9) X(27)
#define GPE_SIZES_p9b(X)
#else
#define GPE_SIZES_p2(X) X(1) X(2) X(4) X(8) X(16) X(32) X(64)
#define GPE_SIZES_p2b(X) X(128) X(256) X(512) X(1024)
#define GPE_SIZES_p3(X) X(3) X(6) X(12) X(24) X(48)
#define GPE_SIZES_p3b(X) X(96) X(192) X(384) X(768)
#define GPE_SIZES_p5(X) X(5) X(10) X(20) X(40) X(80) X(25) X(50)
#define GPE_SIZES_p5b(X) X(160) X(320) X(640) X(100) X(200) X(400) X(800)
#define GPE_SIZES_p9(X) X(9) X(18) X(36) X(72) X(27) X(54)
#define GPE_SIZES_p9b(X) X(144) X(288) X(576) X(108) X(216) X(432) X(864)
#endif
