// treesap-b200 C ABI: scalar wave models with stencil half-width 1.
#define TSB_G 1
#include "models_wave.cuh"
