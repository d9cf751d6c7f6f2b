// XML reader for the reference CLI's scene loader (cli/scene_loader.cpp),
// which is written against pugixml's DOM API (pugixml v1.15, fetched by the
// reference's cli/CMakeLists.txt and not part of this image). This header
// declares the part of that API the loader and this project's tests use, with
// the same names and meaning; xml_reader.cpp implements it with a parser of
// this project's own.
//
// Parsing follows pugixml's default options (parse_default): elements,
// attributes and non-blank text become nodes; character and the five
// predefined entity references are expanded; CDATA sections become cdata
// nodes; the XML declaration, processing instructions, comments and the
// document type declaration are checked for termination and dropped;
// line ends are normalised to '\n' in text and tabs / line ends in attribute
// values become spaces. Handles are non-owning views into the document, and
// a default-constructed (or not-found) handle is empty: its name() and
// value() are "", its lookups return empty handles, and it converts to
// false.
#pragma once

#include <cstddef>
#include <deque>
#include <iterator>
#include <string>
#include <vector>

namespace pugi
{

enum xml_node_type
{
    node_null,
    node_document,
    node_element,
    node_pcdata,
    node_cdata,
    node_comment,
    node_pi,
    node_declaration,
    node_doctype
};

enum xml_parse_status
{
    status_ok = 0,
    status_file_not_found,
    status_io_error,
    status_out_of_memory,
    status_internal_error,
    status_unrecognized_tag,
    status_bad_pi,
    status_bad_comment,
    status_bad_cdata,
    status_bad_doctype,
    status_bad_pcdata,
    status_bad_start_element,
    status_bad_attribute,
    status_bad_end_element,
    status_end_element_mismatch,
    status_append_invalid_root,
    status_no_document_element
};

enum xml_encoding
{
    encoding_auto,
    encoding_utf8
};

// Only the default option set is implemented; the constants exist so calls
// written against pugixml compile.
const unsigned int parse_default = 0x0074u;

namespace impl
{
struct attr_record
{
    std::string name;
    std::string value;
};

struct node_record
{
    xml_node_type type = node_null;
    std::string name;
    std::string value;
    std::vector<attr_record> attributes;
    node_record* parent = nullptr;
    node_record* first_child = nullptr;
    node_record* last_child = nullptr;
    node_record* next_sibling = nullptr;
    node_record* prev_sibling = nullptr;
};
} // namespace impl

class xml_node;

class xml_attribute
{
public:
    xml_attribute() = default;

    explicit operator bool() const { return attr_ != nullptr; }
    bool operator!() const { return attr_ == nullptr; }
    bool operator==(const xml_attribute& o) const { return attr_ == o.attr_; }
    bool operator!=(const xml_attribute& o) const { return attr_ != o.attr_; }

    bool empty() const { return attr_ == nullptr; }
    const char* name() const { return attr_ ? attr_->name.c_str() : ""; }
    const char* value() const { return attr_ ? attr_->value.c_str() : ""; }

    // The next attribute of the same element, or an empty handle.
    xml_attribute next_attribute() const;
    xml_attribute previous_attribute() const;

    // Conversions; the default is returned for an empty handle.
    const char* as_string(const char* def = "") const { return attr_ ? attr_->value.c_str() : def; }
    int as_int(int def = 0) const;
    unsigned int as_uint(unsigned int def = 0) const;
    double as_double(double def = 0) const;
    float as_float(float def = 0) const;
    bool as_bool(bool def = false) const;

private:
    friend class xml_node;
    friend class xml_attribute_iterator;
    xml_attribute(const impl::node_record* owner, const impl::attr_record* attr)
        : owner_(owner)
        , attr_(attr)
    {
    }

    const impl::node_record* owner_ = nullptr;
    const impl::attr_record* attr_ = nullptr;
};

template <typename It>
class xml_object_range
{
public:
    typedef It const_iterator;
    typedef It iterator;

    xml_object_range(It b, It e)
        : begin_(b)
        , end_(e)
    {
    }

    It begin() const { return begin_; }
    It end() const { return end_; }
    bool empty() const { return begin_ == end_; }

private:
    It begin_, end_;
};

class xml_node_iterator;
class xml_named_node_iterator;
class xml_attribute_iterator;

class xml_node
{
public:
    xml_node() = default;

    explicit operator bool() const { return node_ != nullptr; }
    bool operator!() const { return node_ == nullptr; }
    bool operator==(const xml_node& o) const { return node_ == o.node_; }
    bool operator!=(const xml_node& o) const { return node_ != o.node_; }

    bool empty() const { return node_ == nullptr; }
    xml_node_type type() const { return node_ ? node_->type : node_null; }

    // Element name ("" for text, CDATA and the document); text / CDATA
    // content for those nodes ("" for elements).
    const char* name() const { return node_ ? node_->name.c_str() : ""; }
    const char* value() const { return node_ ? node_->value.c_str() : ""; }

    xml_node parent() const { return xml_node(node_ ? node_->parent : nullptr); }
    xml_node first_child() const { return xml_node(node_ ? node_->first_child : nullptr); }
    xml_node last_child() const { return xml_node(node_ ? node_->last_child : nullptr); }
    xml_node next_sibling() const { return xml_node(node_ ? node_->next_sibling : nullptr); }
    xml_node previous_sibling() const { return xml_node(node_ ? node_->prev_sibling : nullptr); }

    // The first child element / next sibling element with this name.
    xml_node child(const char* name) const;
    xml_node next_sibling(const char* name) const;
    xml_node previous_sibling(const char* name) const;

    // The attribute with this name, or an empty handle.
    xml_attribute attribute(const char* name) const;
    xml_attribute first_attribute() const;
    xml_attribute last_attribute() const;

    // Value of the first text or CDATA child ("" when there is none), and of
    // the named child element's first text child.
    const char* child_value() const;
    const char* child_value(const char* name) const;

    xml_object_range<xml_node_iterator> children() const;
    xml_object_range<xml_named_node_iterator> children(const char* name) const;
    xml_object_range<xml_attribute_iterator> attributes() const;

    xml_node_iterator begin() const;
    xml_node_iterator end() const;

protected:
    friend class xml_node_iterator;
    friend class xml_named_node_iterator;
    friend class xml_attribute;
    friend class xml_document;
    explicit xml_node(const impl::node_record* n)
        : node_(n)
    {
    }

    const impl::node_record* node_ = nullptr;
};

class xml_node_iterator
{
public:
    typedef std::ptrdiff_t difference_type;
    typedef xml_node value_type;
    typedef const xml_node* pointer;
    typedef const xml_node& reference;
    typedef std::forward_iterator_tag iterator_category;

    xml_node_iterator() = default;
    explicit xml_node_iterator(const xml_node& n)
        : cur_(n)
    {
    }

    bool operator==(const xml_node_iterator& o) const { return cur_ == o.cur_; }
    bool operator!=(const xml_node_iterator& o) const { return cur_ != o.cur_; }
    const xml_node& operator*() const { return cur_; }
    const xml_node* operator->() const { return &cur_; }
    xml_node_iterator& operator++()
    {
        cur_ = cur_.next_sibling();
        return *this;
    }
    xml_node_iterator operator++(int)
    {
        xml_node_iterator t = *this;
        ++*this;
        return t;
    }

private:
    xml_node cur_;
};

class xml_named_node_iterator
{
public:
    typedef std::ptrdiff_t difference_type;
    typedef xml_node value_type;
    typedef const xml_node* pointer;
    typedef const xml_node& reference;
    typedef std::forward_iterator_tag iterator_category;

    xml_named_node_iterator() = default;
    xml_named_node_iterator(const xml_node& n, const char* name)
        : cur_(n)
        , name_(name)
    {
    }

    bool operator==(const xml_named_node_iterator& o) const { return cur_ == o.cur_; }
    bool operator!=(const xml_named_node_iterator& o) const { return cur_ != o.cur_; }
    const xml_node& operator*() const { return cur_; }
    const xml_node* operator->() const { return &cur_; }
    xml_named_node_iterator& operator++()
    {
        cur_ = cur_.next_sibling(name_);
        return *this;
    }
    xml_named_node_iterator operator++(int)
    {
        xml_named_node_iterator t = *this;
        ++*this;
        return t;
    }

private:
    xml_node cur_;
    const char* name_ = "";
};

class xml_attribute_iterator
{
public:
    typedef std::ptrdiff_t difference_type;
    typedef xml_attribute value_type;
    typedef const xml_attribute* pointer;
    typedef const xml_attribute& reference;
    typedef std::forward_iterator_tag iterator_category;

    xml_attribute_iterator() = default;
    explicit xml_attribute_iterator(const xml_attribute& a)
        : cur_(a)
    {
    }

    bool operator==(const xml_attribute_iterator& o) const { return cur_ == o.cur_; }
    bool operator!=(const xml_attribute_iterator& o) const { return cur_ != o.cur_; }
    const xml_attribute& operator*() const { return cur_; }
    const xml_attribute* operator->() const { return &cur_; }
    xml_attribute_iterator& operator++()
    {
        cur_ = cur_.next_attribute();
        return *this;
    }
    xml_attribute_iterator operator++(int)
    {
        xml_attribute_iterator t = *this;
        ++*this;
        return t;
    }

private:
    xml_attribute cur_;
};

struct xml_parse_result
{
    xml_parse_status status = status_internal_error;
    std::ptrdiff_t offset = 0; // byte offset of the error in the input
    xml_encoding encoding = encoding_utf8;

    explicit operator bool() const { return status == status_ok; }
    bool operator!() const { return status != status_ok; }
    const char* description() const;
};

// Owns the parsed tree; the handles it hands out stay valid until the next
// load or reset, or the document's destruction.
class xml_document : public xml_node
{
public:
    xml_document();
    xml_document(const xml_document&) = delete;
    xml_document& operator=(const xml_document&) = delete;

    void reset();

    xml_parse_result load_file(const char* path, unsigned int options = parse_default,
                               xml_encoding encoding = encoding_auto);
    xml_parse_result load_string(const char* contents, unsigned int options = parse_default);
    xml_parse_result load_buffer(const void* contents, std::size_t size, unsigned int options = parse_default,
                                 xml_encoding encoding = encoding_auto);

    // The root element, or an empty handle.
    xml_node document_element() const;

private:
    std::deque<impl::node_record> nodes_; // nodes_[0] is the document node
};

} // namespace pugi
