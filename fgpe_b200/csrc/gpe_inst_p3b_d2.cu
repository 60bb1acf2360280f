// Pass-kernel instantiations: length family p3b, double, 2 field(s) per pass.
#include "gpe_sizes.h"
#define GPE_R double
#define GPE_SFX d
#define GPE_FAM p3b
#define GPE_NF 2
#define GPE_SIZES(X) GPE_SIZES_p3b(X)
#define GPE_TUNED(X) GPE_TUNED_p3b(X)
#include "gpe_inst_body.cuh"
