// Pass-kernel instantiations: length family p9, float, 1 field(s) per pass.
#include "gpe_sizes.h"
#define GPE_R float
#define GPE_PAIRED 1
#define GPE_SFX f
#define GPE_FAM p9
#define GPE_NF 1
#define GPE_SIZES(X) GPE_SIZES_p9(X)
#define GPE_TUNED(X) GPE_TUNED_p9(X)
#include "gpe_inst_body.cuh"
