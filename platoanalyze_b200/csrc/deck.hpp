// Input decks: a small XML reader and the typed parameter tree of Teuchos::ParameterList
// XML (the format of the reference's input configs, e.g. `<ParameterList name='Plato
// Problem'> <Parameter name='Physics' type='string' value='Mechanical'/> ...`), plus the
// element-text form PlatoEngine application files use (`<Operation> <Function>...`).
// Host code only; errors throw DeckError, which the C ABI turns into PLATO_BAD_INPUT.
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace plato::deck {

struct DeckError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

struct XmlNode {
    std::string tag;
    std::vector<std::pair<std::string, std::string>> attrs;
    std::vector<XmlNode> children;
    std::string text;  // concatenated character data directly inside the element, trimmed

    const std::string* attr(const std::string& name) const;
    std::vector<const XmlNode*> children_named(const std::string& tag) const;
    // text of the first child element `tag`, or `fallback` when there is none
    std::string child_text(const std::string& tag, const std::string& fallback = std::string()) const;
    bool has_child(const std::string& tag) const;
};

// Parses a document (XML declaration, comments and processing instructions skipped, the five
// predefined entities and numeric character references decoded) and returns its root.
// Several top-level elements are wrapped in one root with an empty tag.
XmlNode parse_xml(const std::string& text);

struct ParamList;

struct ParamEntry {
    std::string type;   // Teuchos type name: double, int, bool, string, Array(double), ...
    std::string value;  // the value attribute as written
    std::shared_ptr<ParamList> list;  // set for a sublist
    bool is_list() const { return static_cast<bool>(list); }
};

// Teuchos::ParameterList: named entries in insertion order; a name occurs once per list.
struct ParamList {
    std::string name;
    std::vector<std::pair<std::string, ParamEntry>> entries;

    const ParamEntry* find(const std::string& key) const;
    bool has(const std::string& key) const { return find(key) != nullptr; }
    bool is_sublist(const std::string& key) const;
    const ParamList& sublist(const std::string& key) const;  // throws when absent

    std::string get_string(const std::string& key) const;
    std::string get_string(const std::string& key, const std::string& fallback) const;
    double get_double(const std::string& key) const;
    double get_double(const std::string& key, double fallback) const;
    int get_int(const std::string& key) const;
    int get_int(const std::string& key, int fallback) const;
    bool get_bool(const std::string& key, bool fallback) const;
    std::vector<double> get_double_array(const std::string& key) const;      // "{1.0, 2.0}"
    std::vector<std::string> get_string_array(const std::string& key) const;  // "{a, b}"
    bool is_type(const std::string& key, const std::string& type) const;

    // Sets a double at an operation parameter's Target: ':'-separated tokens, leading tokens
    // in brackets name sublists that must exist ("[Plato Problem]:[Criteria]:[Energy]:Exponent"),
    // the last token is a parameter name (created when absent) or "Name(i)", entry i of an
    // existing Array(double).
    void set_target(const std::string& target, double value);
};

// The ParameterList element at `root` (or its first ParameterList descendant when `root`
// is a wrapper) as a tree.
std::shared_ptr<ParamList> to_param_list(const XmlNode& root);
std::shared_ptr<ParamList> parse_param_list(const std::string& xml_text);

// Reads a whole file; throws DeckError when it cannot be opened.
std::string read_file(const std::string& path);

}  // namespace plato::deck
