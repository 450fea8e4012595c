// ScannerHeader of FIR's public headers: declared with ScannerData in ScannerData.h.
#pragma once

#include <ScannerData.h>
