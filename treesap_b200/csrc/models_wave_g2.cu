// treesap-b200 C ABI: scalar wave models with stencil half-width 2.
#define TSB_G 2
#include "models_wave.cuh"
