// treesap-b200 C ABI: scalar wave models with stencil half-width 4.
#define TSB_G 4
#include "models_wave.cuh"
