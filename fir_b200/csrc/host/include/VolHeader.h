// VolHeader of FIR's public headers: declared with VolData in VolData.h.
#pragma once

#include <VolData.h>
