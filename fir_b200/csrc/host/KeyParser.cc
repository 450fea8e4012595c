// Interfile-style key parser (see KeyParser.h for the rules, which follow
// FIR's src_lib/KeyParser.cc).
#include <KeyParser.h>
#include <console.h>

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace
{
const char* kBlank = " \t";

std::string substituteEnv(std::string s)
{
  std::string::size_type at;
  while ((at = s.find("${")) != std::string::npos)
  {
    const auto close = s.find('}', at + 2);
    if (close == std::string::npos)
    {
      break;
    }
    const auto name = s.substr(at + 2, close - at - 2);
    const char* value = std::getenv(name.c_str());
    if (value == nullptr)
    {
      warning("Environment variable '", name, " not found. Replaced by empty string.\n",
              "This happened on the following line: ", s);
      s.erase(at, close - at + 1);
    }
    else
    {
      s.replace(at, close - at + 1, value);
    }
  }
  return s;
}

// Text after the first '=', or npos if none / nothing after it.
std::string::size_type valueStart(const std::string& line)
{
  const auto eq = line.find('=');
  if (eq == std::string::npos)
  {
    return std::string::npos;
  }
  return line.find_first_not_of(kBlank, eq + 1);
}

template<typename T>
bool scalar(const std::string& line, T& out)
{
  const auto eq = line.find('=');
  if (eq == std::string::npos)
  {
    return false;
  }
  std::istringstream is(line.substr(eq + 1));
  T v{};
  is >> v;
  if (is.fail())
  {
    return false;
  }
  out = v;
  return true;
}

template<typename T>
bool list(const std::string& line, std::vector<T>& out)
{
  const auto start = valueStart(line);
  if (start == std::string::npos)
  {
    return false;
  }
  std::istringstream is(line.substr(start));
  std::vector<T> values;
  if (line[start] != '{')
  {
    T v{};
    is >> v;
    if (is.fail())
    {
      return false;
    }
    out.assign(1, v);
    return true;
  }
  char c;
  is >> c;  // '{'
  while (true)
  {
    T v{};
    is >> v;
    if (is.fail())
    {
      is.clear();
      break;
    }
    values.push_back(v);
    is >> std::ws >> c;
    if (is.fail() || c != ',')
    {
      break;
    }
  }
  if (c != '}')
  {
    is >> std::ws >> c;
    if (is.fail() || c != '}')
    {
      warning("While reading a vector, expected closing }. Length of vector returned is ", values.size());
    }
  }
  out = values;
  return true;
}
}  // namespace

std::string KeyParser::standardiseKeyword(const std::string& keyword)
{
  const char* ws = " \t_!";
  const auto first = keyword.find_first_not_of(ws);
  if (first == std::string::npos)
  {
    return {};
  }
  const auto last = keyword.find_last_not_of(ws);
  std::string out;
  bool prevBlank = false;
  for (auto i = first; i <= last; ++i)
  {
    const char ch = keyword[i];
    if (std::isspace(static_cast<unsigned char>(ch)) || ch == '_' || ch == '!')
    {
      if (!prevBlank)
      {
        out += ' ';
        prevBlank = true;
      }
      continue;
    }
    if (ch == '[' && !prevBlank)
    {
      out += " [";
    }
    else
    {
      out += static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
    }
    prevBlank = false;
  }
  return out;
}

void KeyParser::add(const std::string& keyword, Kind kind, void* target)
{
  const auto key = standardiseKeyword(keyword);
  for (auto& e : mEntries)
  {
    if (e.key == key)
    {
      warning("Keyword ", keyword, " already registered for parsing. Overwriting previous value.");
      e = Entry{key, kind, target};
      return;
    }
  }
  mEntries.push_back(Entry{key, kind, target});
}

void KeyParser::addStartKey(const std::string& k) { add(k, Kind::Start, nullptr); }
void KeyParser::addStopKey(const std::string& k) { add(k, Kind::Stop, nullptr); }
void KeyParser::addKey(const std::string& k, std::string* p) { add(k, Kind::Ascii, p); }
void KeyParser::addKey(const std::string& k, int* p) { add(k, Kind::Int, p); }
void KeyParser::addKey(const std::string& k, float* p) { add(k, Kind::Float, p); }
void KeyParser::addKey(const std::string& k, double* p) { add(k, Kind::Double, p); }
void KeyParser::addKey(const std::string& k, std::vector<int>* p) { add(k, Kind::Ints, p); }
void KeyParser::addKey(const std::string& k, std::vector<float>* p) { add(k, Kind::Floats, p); }
void KeyParser::addKey(const std::string& k, std::vector<double>* p) { add(k, Kind::Doubles, p); }

const KeyParser::Entry* KeyParser::find(const std::string& key) const
{
  for (const auto& e : mEntries)
  {
    if (e.key == key)
    {
      return &e;
    }
  }
  return nullptr;
}

bool KeyParser::assign(const Entry& e, const std::string& line)
{
  switch (e.kind)
  {
  case Kind::Ascii:
  {
    const auto start = valueStart(line);
    if (start == std::string::npos)
    {
      return false;
    }
    const auto stop = line.find_last_not_of(kBlank) + 1;
    *static_cast<std::string*>(e.target) = line.substr(start, stop - start);
    return true;
  }
  case Kind::Int: return scalar(line, *static_cast<int*>(e.target));
  case Kind::Float: return scalar(line, *static_cast<float*>(e.target));
  case Kind::Double: return scalar(line, *static_cast<double*>(e.target));
  case Kind::Ints: return list(line, *static_cast<std::vector<int>*>(e.target));
  case Kind::Floats: return list(line, *static_cast<std::vector<float>*>(e.target));
  case Kind::Doubles: return list(line, *static_cast<std::vector<double>*>(e.target));
  default: return false;
  }
}

bool KeyParser::parse(const std::string& filePath, bool writeWarnings)
{
  std::ifstream in(filePath);
  if (!in)
  {
    error("Couldn't open file ", filePath);
  }
  bool started = false;
  std::string line;
  while (true)
  {
    if (!std::getline(in, line))
    {
      if (started)
      {
        warning("Early EOF or bad file");
      }
      break;
    }
    if (line.find_first_not_of(kBlank) == std::string::npos)
    {
      continue;
    }
    line = substituteEnv(line);
    const auto key = standardiseKeyword(line.substr(0, line.find(':')));
    const Entry* e = find(key);
    if (!started)
    {
      if (e != nullptr && e->kind == Kind::Start)
      {
        started = true;
        continue;
      }
      for (const auto& x : mEntries)
      {
        if (x.kind == Kind::Start)
        {
          warning("Required first keyword \"", x.key, "\" not found");
          return false;
        }
      }
      warning("Data found, but key parser status is \"not parsing\". Keymap possibly incorrect.");
      return false;
    }
    if (e == nullptr)
    {
      if (writeWarnings && !key.empty() && key[0] != ';')
      {
        warning("Unrecognized keyword: ", key);
      }
      continue;
    }
    if (e->kind == Kind::Stop)
    {
      break;
    }
    if (e->kind == Kind::Start)
    {
      continue;
    }
    assign(*e, line);
  }
  return started;
}
