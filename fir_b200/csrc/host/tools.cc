// Utilities of FIR's tools.h (src_lib/tools.cc:17-58).
#include <tools.h>

#include <cctype>
#include <thread>

std::string strToUpper(const std::string& in)
{
  std::string out(in);
  for (auto& c : out)
  {
    c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
  }
  return out;
}

bool systemIsLittleEndian()
{
  const int n = 1;
  return *reinterpret_cast<const char*>(&n) == 1;
}

void addPath(const std::string& headerFile, std::string& dataFile)
{
  if (!dataFile.empty() && dataFile[0] != '/')
  {
    const auto slash = headerFile.find_last_of('/');
    if (slash != std::string::npos)
    {
      dataFile.insert(0, headerFile, 0, slash + 1);
    }
  }
}

int getNThreads()
{
  const unsigned n = std::thread::hardware_concurrency();
  return n > 0 ? static_cast<int>(n) : 1;
}

int getCurrentThread() { return 0; }
