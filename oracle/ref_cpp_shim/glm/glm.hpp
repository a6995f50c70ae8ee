// Stands in for the header of the same name (not part of the reference tree): see ref_cpp_shim.h.
#pragma once
#include "../ref_cpp_shim.h"
