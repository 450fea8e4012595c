// Interfile-style "key := value" parser with FIR's public interface
// (src_lib/KeyParser.h:42-72) and FIR's rules (src_lib/KeyParser.cc):
//   - the first non-empty line must be the start key; parsing stops at the
//     stop key (or at end of file, with a warning);
//   - keywords are the text before the first ':' and are compared after
//     Interfile 3.3 standardisation: space, tab, '_' and '!' are white space,
//     leading/trailing white space is dropped, runs collapse to one space,
//     case is ignored, and "[" is preceded by a space;
//   - values are the text after the first '='; ${NAME} is replaced by the
//     environment variable NAME; lists are written {a, b, c} (a bare value is
//     a list of one);
//   - a key without a value leaves its variable unchanged.
#pragma once

#include <string>
#include <vector>

class KeyParser
{
public:
  KeyParser() = default;

  void addStartKey(const std::string& keyword);
  void addStopKey(const std::string& keyword);

  void addKey(const std::string& keyword, std::string* pVariable);
  void addKey(const std::string& keyword, int* pVariable);
  void addKey(const std::string& keyword, float* pVariable);
  void addKey(const std::string& keyword, double* pVariable);
  void addKey(const std::string& keyword, std::vector<int>* pVariable);
  void addKey(const std::string& keyword, std::vector<float>* pVariable);
  void addKey(const std::string& keyword, std::vector<double>* pVariable);

  // Returns false if the first keyword is not the start key.  Throws (via
  // error()) if the file cannot be opened.
  bool parse(const std::string& filePath, bool writeWarnings = false);

  static std::string standardiseKeyword(const std::string& keyword);

private:
  enum class Kind
  {
    Start,
    Stop,
    Ascii,
    Int,
    Float,
    Double,
    Ints,
    Floats,
    Doubles
  };

  struct Entry
  {
    std::string key;
    Kind kind;
    void* target;
  };

  void add(const std::string& keyword, Kind kind, void* target);
  const Entry* find(const std::string& key) const;
  static bool assign(const Entry& e, const std::string& line);

  std::vector<Entry> mEntries;
};
