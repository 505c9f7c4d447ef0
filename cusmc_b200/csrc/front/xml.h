// Minimal XML reader for UPPAAL model files.
//
// Covers what the UPPAAL flat-system format uses: elements, attributes,
// character data, CDATA, comments, processing instructions and DOCTYPE, and
// the five predefined entities plus numeric character references.  It follows
// the text conventions that the reference's XML library applies by default
// (pugixml parse_default, as called from automata_parser/uppaal_xml_parser.cpp:630):
//   * "\r\n" and "\r" become "\n" everywhere;
//   * tab, newline and carriage return inside attribute values become spaces;
//   * character data consisting only of whitespace is dropped, other
//     character data is kept verbatim (no trimming);
//   * child_value() is the text of the first character-data child.
#pragma once
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace csmc {

struct XmlNode {
    std::string name;                                        // element name
    std::vector<std::pair<std::string, std::string>> attrs;  // in document order
    std::vector<std::unique_ptr<XmlNode>> children;          // elements and text nodes
    bool is_text = false;                                    // character data node
    std::string text;                                        // for text nodes

    // First child element with this name, or nullptr.
    const XmlNode *child(const std::string &n) const;
    // All child elements with this name, in document order.
    std::vector<const XmlNode *> children_named(const std::string &n) const;
    // Attribute value or "" when absent.
    std::string attr(const std::string &n) const;
    bool has_attr(const std::string &n) const;
    // Text of the first character-data child ("" when none).
    std::string child_value() const;
    // child(n)->child_value(), or "" when the child is absent.
    std::string child_text(const std::string &n) const;
};

// Parses a whole document; throws std::runtime_error with a message on
// malformed input.  The returned node is a synthetic root whose children are
// the top-level elements.
std::unique_ptr<XmlNode> xml_parse(const std::string &text);
std::unique_ptr<XmlNode> xml_parse_file(const std::string &path);

}  // namespace csmc
