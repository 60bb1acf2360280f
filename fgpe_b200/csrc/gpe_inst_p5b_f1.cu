// Pass-kernel instantiations: length family p5b, float, 1 field(s) per pass.
#include "gpe_sizes.h"
#define GPE_R float
#define GPE_PAIRED 1
#define GPE_SFX f
#define GPE_FAM p5b
#define GPE_NF 1
#define GPE_SIZES(X) GPE_SIZES_p5b(X)
#define GPE_TUNED(X) GPE_TUNED_p5b(X)
#include "gpe_inst_body.cuh"
