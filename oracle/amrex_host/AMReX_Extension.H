// Forwarding header of the oracle host AMReX-API shim.
#pragma once
#include "amrex_host.H"
