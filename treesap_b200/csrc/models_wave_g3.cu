// treesap-b200 C ABI: scalar wave models with stencil half-width 3.
#define TSB_G 3
#include "models_wave.cuh"
