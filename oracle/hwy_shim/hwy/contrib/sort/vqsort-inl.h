// Stand-in: VQSort/VQSortStatic are provided by hwy/highway.h.
#pragma once
#include "hwy/highway.h"
