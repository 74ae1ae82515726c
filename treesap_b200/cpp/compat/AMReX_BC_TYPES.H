// treesap-b200 amrex compatibility layer: forwarding header.
#pragma once
#include "AMReX.H"
