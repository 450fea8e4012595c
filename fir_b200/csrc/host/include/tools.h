// Small utilities of FIR's public headers (src_lib/tools.h:1-33).
#pragma once

#include <algorithm>
#include <cstring>
#include <string>

std::string strToUpper(const std::string& in);
bool systemIsLittleEndian();
// Prepends the directory of headerFile to a relative dataFile (in place)
void addPath(const std::string& headerFile, std::string& dataFile);
// Host threads available to the process (the GPU does the projection work)
int getNThreads();
int getCurrentThread();

template<typename T>
T swapEndianness(T u)
{
  unsigned char b[sizeof(T)];
  std::memcpy(b, &u, sizeof(T));
  std::reverse(b, b + sizeof(T));
  std::memcpy(&u, b, sizeof(T));
  return u;
}
