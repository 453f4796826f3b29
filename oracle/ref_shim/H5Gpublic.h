// TEST INFRASTRUCTURE ONLY: stand-in for the HDF5 header of this name (see h5_stub.h).
#pragma once
#include "h5_stub.h"
