#pragma once
#include "tbb_ordered_shim.h"
