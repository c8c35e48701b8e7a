// Minimal XML reader for MJCF: elements, attributes, comments, <?...?> and
// CDATA-free text.  Enough for the MJCF subset the model compiler accepts.
#pragma once
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace mjb {

struct XmlNode {
  std::string tag;
  std::vector<std::pair<std::string, std::string>> attrs;
  std::vector<XmlNode> children;
  int line = 0;

  const std::string* attr(const char* name) const {
    for (auto& kv : attrs)
      if (kv.first == name) return &kv.second;
    return nullptr;
  }
};

// Parses one XML document; throws std::runtime_error with the line number on
// malformed input.
XmlNode parse_xml(const std::string& text);

}  // namespace mjb
