// ProjHeader of FIR's public headers: declared with ProjData in ProjData.h.
#pragma once

#include <ProjData.h>
