// Stand-in: VQSort is provided by hwy/highway.h.
#pragma once
#include "hwy/highway.h"
