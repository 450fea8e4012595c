// Console helpers of FIR's public headers (src_lib/console.h, console.inl):
// progress printing and error(), which throws std::runtime_error whose text
// starts with "ERROR: " and ends with a newline, as FIR's does.
#pragma once

#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

inline void echo(const std::string& message) { std::cout << message << std::endl; }

template<typename... Args>
void print(Args&&... args)
{
  std::stringstream m;
  ((m << std::forward<Args>(args)), ...);
  m << std::endl;
  std::cout << m.str();
}

template<typename T>
void printValue(const std::string& name, const T& value)
{
  std::cout << name << ": " << value << std::endl;
}

template<typename T>
void printQuotedValue(const std::string& name, const T& value)
{
  std::cout << name << ": \"" << value << "\"" << std::endl;
}

template<typename T>
void printVector(const std::string& name, const std::vector<T>& values)
{
  std::cout << name << ": { ";
  for (size_t i = 0; i < values.size(); ++i)
  {
    std::cout << (i ? ", " : "") << values[i];
  }
  std::cout << " }" << std::endl;
}

inline void printEmptyLine() { std::cout << std::endl; }

template<typename... Args>
void warning(Args&&... args)
{
  std::stringstream m;
  m << "WARNING: ";
  ((m << std::forward<Args>(args)), ...);
  m << std::endl;
  std::cout << m.str();
}

template<typename... Args>
[[noreturn]] void error(Args&&... args)
{
  std::stringstream m;
  m << "ERROR: ";
  ((m << std::forward<Args>(args)), ...);
  m << std::endl;
  throw std::runtime_error(m.str());
}
