#pragma once
#include "tbb_serial_shim.h"
