// The XML reader behind pugixml.hpp: a single-pass parser with an explicit
// cursor (no recursion, so nesting depth is bounded only by memory) that
// builds the node tree of an in-memory document (UTF-8; a leading byte-order
// mark is skipped). Every construct is checked for its terminator, and the
// first error stops the parse with pugixml's status for it and the byte
// offset where it was found; the nodes read up to then stay in the document.

#include "pugixml.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

namespace pugi
{

namespace
{

using impl::attr_record;
using impl::node_record;

bool IsSpace(unsigned char c)
{
    return c == ' ' || c == '\t' || c == '\n' || c == '\r';
}

// Name characters as pugixml classifies them: letters, '_' and ':' (and any
// byte of a multi-byte UTF-8 sequence) may start a name; digits, '-' and '.'
// may follow.
bool IsNameStart(unsigned char c)
{
    return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '_' || c == ':' || c >= 0x80;
}

bool IsNameChar(unsigned char c)
{
    return IsNameStart(c) || (c >= '0' && c <= '9') || c == '-' || c == '.';
}

void AppendUtf8(std::string& out, unsigned long cp)
{
    if (cp < 0x80)
    {
        out += char(cp);
    }
    else if (cp < 0x800)
    {
        out += char(0xC0 | (cp >> 6));
        out += char(0x80 | (cp & 0x3F));
    }
    else if (cp < 0x10000)
    {
        out += char(0xE0 | (cp >> 12));
        out += char(0x80 | ((cp >> 6) & 0x3F));
        out += char(0x80 | (cp & 0x3F));
    }
    else
    {
        out += char(0xF0 | (cp >> 18));
        out += char(0x80 | ((cp >> 12) & 0x3F));
        out += char(0x80 | ((cp >> 6) & 0x3F));
        out += char(0x80 | (cp & 0x3F));
    }
}

// Expands one entity reference starting at s[0] == '&' into out and returns
// the characters consumed; 0 when the text there is not a well-formed
// reference (the '&' is then kept as it is).
size_t ExpandEntity(const char* s, const char* end, std::string& out)
{
    const char* semi = static_cast<const char*>(std::memchr(s, ';', size_t(end - s)));
    if (!semi || semi - s > 12)
    {
        return 0;
    }
    std::string ref(s + 1, semi);
    static const struct
    {
        const char* name;
        char ch;
    } kNamed[] = { { "lt", '<' }, { "gt", '>' }, { "amp", '&' }, { "quot", '"' }, { "apos", '\'' } };
    for (const auto& e : kNamed)
    {
        if (ref == e.name)
        {
            out += e.ch;
            return size_t(semi - s) + 1;
        }
    }
    if (ref.size() >= 2 && ref[0] == '#')
    {
        bool hex = ref[1] == 'x';
        const char* digits = ref.c_str() + (hex ? 2 : 1);
        if (*digits == '\0')
        {
            return 0;
        }
        char* stop = nullptr;
        unsigned long cp = std::strtoul(digits, &stop, hex ? 16 : 10);
        if (*stop != '\0' || cp > 0x10FFFF)
        {
            return 0;
        }
        AppendUtf8(out, cp);
        return size_t(semi - s) + 1;
    }
    return 0;
}

class Parser
{
public:
    Parser(std::deque<node_record>& nodes, const char* data, size_t size)
        : nodes_(nodes)
        , begin_(data)
        , s_(data)
        , end_(data + size)
    {
    }

    xml_parse_result Run()
    {
        if (end_ - s_ >= 3 && std::memcmp(s_, "\xEF\xBB\xBF", 3) == 0)
        {
            s_ += 3;
        }
        node_record* cursor = &nodes_.front();
        while (s_ < end_)
        {
            if (*s_ != '<')
            {
                Text(cursor);
                continue;
            }
            xml_parse_status st = Markup(cursor);
            if (st != status_ok)
            {
                return Result(st);
            }
        }
        if (cursor != &nodes_.front())
        {
            return Result(status_end_element_mismatch);
        }
        for (const node_record* c = nodes_.front().first_child; c; c = c->next_sibling)
        {
            if (c->type == node_element)
            {
                return Result(status_ok, true);
            }
        }
        return Result(status_no_document_element);
    }

private:
    xml_parse_result Result(xml_parse_status st, bool ok_offset_zero = false)
    {
        xml_parse_result r;
        r.status = st;
        r.offset = ok_offset_zero ? 0 : (s_ - begin_);
        r.encoding = encoding_utf8;
        return r;
    }

    bool StartsWith(const char* lit) const
    {
        size_t n = std::strlen(lit);
        return size_t(end_ - s_) >= n && std::memcmp(s_, lit, n) == 0;
    }

    const char* Find(const char* from, const char* lit) const
    {
        size_t n = std::strlen(lit);
        for (const char* p = from; p + n <= end_; ++p)
        {
            if (std::memcmp(p, lit, n) == 0)
            {
                return p;
            }
        }
        return nullptr;
    }

    node_record* Append(node_record* parent, xml_node_type type)
    {
        nodes_.emplace_back();
        node_record* n = &nodes_.back();
        n->type = type;
        n->parent = parent;
        n->prev_sibling = parent->last_child;
        if (parent->last_child)
        {
            parent->last_child->next_sibling = n;
        }
        else
        {
            parent->first_child = n;
        }
        parent->last_child = n;
        return n;
    }

    // Character data up to the next '<': kept as a text node unless it is all
    // blank; "\r\n" and a lone '\r' become '\n', entity references expand.
    void Text(node_record* cursor)
    {
        const char* stop = static_cast<const char*>(std::memchr(s_, '<', size_t(end_ - s_)));
        if (!stop)
        {
            stop = end_;
        }
        bool blank = true;
        for (const char* p = s_; p < stop; ++p)
        {
            if (!IsSpace(static_cast<unsigned char>(*p)))
            {
                blank = false;
                break;
            }
        }
        if (!blank)
        {
            std::string text;
            text.reserve(size_t(stop - s_));
            for (const char* p = s_; p < stop;)
            {
                if (*p == '&')
                {
                    size_t used = ExpandEntity(p, stop, text);
                    if (used)
                    {
                        p += used;
                        continue;
                    }
                }
                if (*p == '\r')
                {
                    text += '\n';
                    p += (p + 1 < stop && p[1] == '\n') ? 2 : 1;
                    continue;
                }
                text += *p++;
            }
            Append(cursor, node_pcdata)->value = std::move(text);
        }
        s_ = stop;
    }

    xml_parse_status Markup(node_record*& cursor)
    {
        if (StartsWith("<?"))
        {
            // Declaration or processing instruction: dropped.
            const char* close = Find(s_ + 2, "?>");
            if (!close)
            {
                return status_bad_pi;
            }
            s_ = close + 2;
            return status_ok;
        }
        if (StartsWith("<!--"))
        {
            const char* close = Find(s_ + 4, "-->");
            if (!close)
            {
                return status_bad_comment;
            }
            s_ = close + 3;
            return status_ok;
        }
        if (StartsWith("<![CDATA["))
        {
            const char* close = Find(s_ + 9, "]]>");
            if (!close)
            {
                return status_bad_cdata;
            }
            std::string text;
            for (const char* p = s_ + 9; p < close;)
            {
                if (*p == '\r')
                {
                    text += '\n';
                    p += (p + 1 < close && p[1] == '\n') ? 2 : 1;
                    continue;
                }
                text += *p++;
            }
            Append(cursor, node_cdata)->value = std::move(text);
            s_ = close + 3;
            return status_ok;
        }
        if (StartsWith("<!DOCTYPE"))
        {
            return Doctype();
        }
        if (StartsWith("</"))
        {
            return EndTag(cursor);
        }
        if (end_ - s_ >= 2 && IsNameStart(static_cast<unsigned char>(s_[1])))
        {
            return StartTag(cursor);
        }
        return status_unrecognized_tag;
    }

    // <!DOCTYPE ...> with an optional internal subset in brackets, whose
    // quoted strings and nested declarations may contain '>'.
    xml_parse_status Doctype()
    {
        int depth = 0;
        for (const char* p = s_ + 9; p < end_; ++p)
        {
            char c = *p;
            if (c == '"' || c == '\'')
            {
                const char* q = static_cast<const char*>(std::memchr(p + 1, c, size_t(end_ - p - 1)));
                if (!q)
                {
                    return status_bad_doctype;
                }
                p = q;
            }
            else if (c == '[')
            {
                ++depth;
            }
            else if (c == ']')
            {
                --depth;
            }
            else if (c == '>' && depth <= 0)
            {
                s_ = p + 1;
                return status_ok;
            }
        }
        return status_bad_doctype;
    }

    std::string Name()
    {
        const char* start = s_;
        while (s_ < end_ && IsNameChar(static_cast<unsigned char>(*s_)))
        {
            ++s_;
        }
        return std::string(start, s_);
    }

    void SkipSpace()
    {
        while (s_ < end_ && IsSpace(static_cast<unsigned char>(*s_)))
        {
            ++s_;
        }
    }

    xml_parse_status StartTag(node_record*& cursor)
    {
        ++s_; // '<'
        node_record* element = Append(cursor, node_element);
        element->name = Name();
        if (s_ >= end_ || !(IsSpace(static_cast<unsigned char>(*s_)) || *s_ == '/' || *s_ == '>'))
        {
            return status_bad_start_element;
        }
        for (;;)
        {
            bool spaced = s_ < end_ && IsSpace(static_cast<unsigned char>(*s_));
            SkipSpace();
            if (s_ >= end_)
            {
                return status_bad_start_element;
            }
            if (*s_ == '>')
            {
                ++s_;
                cursor = element;
                return status_ok;
            }
            if (*s_ == '/')
            {
                if (s_ + 1 >= end_ || s_[1] != '>')
                {
                    return status_bad_start_element;
                }
                s_ += 2;
                return status_ok;
            }
            if (!spaced || !IsNameStart(static_cast<unsigned char>(*s_)))
            {
                return status_bad_attribute;
            }
            attr_record attr;
            attr.name = Name();
            SkipSpace();
            if (s_ >= end_ || *s_ != '=')
            {
                return status_bad_attribute;
            }
            ++s_;
            SkipSpace();
            if (s_ >= end_ || (*s_ != '"' && *s_ != '\''))
            {
                return status_bad_attribute;
            }
            char quote = *s_++;
            const char* close = static_cast<const char*>(std::memchr(s_, quote, size_t(end_ - s_)));
            if (!close)
            {
                return status_bad_attribute;
            }
            for (const char* p = s_; p < close;)
            {
                if (*p == '&')
                {
                    size_t used = ExpandEntity(p, close, attr.value);
                    if (used)
                    {
                        p += used;
                        continue;
                    }
                }
                if (*p == '\r' || *p == '\n' || *p == '\t')
                {
                    attr.value += ' ';
                    p += (*p == '\r' && p + 1 < close && p[1] == '\n') ? 2 : 1;
                    continue;
                }
                attr.value += *p++;
            }
            element->attributes.push_back(std::move(attr));
            s_ = close + 1;
        }
    }

    xml_parse_status EndTag(node_record*& cursor)
    {
        const char* at = s_;
        s_ += 2;
        std::string name = Name();
        SkipSpace();
        if (s_ >= end_ || *s_ != '>')
        {
            return status_bad_end_element;
        }
        if (cursor->type != node_element || cursor->name != name)
        {
            s_ = at;
            return status_end_element_mismatch;
        }
        ++s_;
        cursor = cursor->parent;
        return status_ok;
    }

    std::deque<node_record>& nodes_;
    const char* begin_;
    const char* s_;
    const char* end_;
};

const node_record* FindChild(const node_record* first, const char* name)
{
    for (const node_record* c = first; c; c = c->next_sibling)
    {
        if (c->type == node_element && c->name == name)
        {
            return c;
        }
    }
    return nullptr;
}

} // namespace

// ------------------------------------------------------------ xml_attribute

xml_attribute xml_attribute::next_attribute() const
{
    if (!attr_)
    {
        return xml_attribute();
    }
    const auto& all = owner_->attributes;
    size_t i = size_t(attr_ - all.data()) + 1;
    return i < all.size() ? xml_attribute(owner_, &all[i]) : xml_attribute();
}

xml_attribute xml_attribute::previous_attribute() const
{
    if (!attr_)
    {
        return xml_attribute();
    }
    const auto& all = owner_->attributes;
    size_t i = size_t(attr_ - all.data());
    return i > 0 ? xml_attribute(owner_, &all[i - 1]) : xml_attribute();
}

int xml_attribute::as_int(int def) const
{
    if (!attr_)
    {
        return def;
    }
    return int(std::strtol(attr_->value.c_str(), nullptr, 0));
}

unsigned int xml_attribute::as_uint(unsigned int def) const
{
    if (!attr_)
    {
        return def;
    }
    return unsigned(std::strtoul(attr_->value.c_str(), nullptr, 0));
}

double xml_attribute::as_double(double def) const
{
    return attr_ ? std::strtod(attr_->value.c_str(), nullptr) : def;
}

float xml_attribute::as_float(float def) const
{
    return attr_ ? std::strtof(attr_->value.c_str(), nullptr) : def;
}

bool xml_attribute::as_bool(bool def) const
{
    if (!attr_)
    {
        return def;
    }
    char c = attr_->value.empty() ? '\0' : attr_->value[0];
    return c == '1' || c == 't' || c == 'T' || c == 'y' || c == 'Y';
}

// ----------------------------------------------------------------- xml_node

xml_node xml_node::child(const char* name) const
{
    return xml_node(node_ ? FindChild(node_->first_child, name) : nullptr);
}

xml_node xml_node::next_sibling(const char* name) const
{
    return xml_node(node_ ? FindChild(node_->next_sibling, name) : nullptr);
}

xml_node xml_node::previous_sibling(const char* name) const
{
    for (const node_record* c = node_ ? node_->prev_sibling : nullptr; c; c = c->prev_sibling)
    {
        if (c->type == node_element && c->name == name)
        {
            return xml_node(c);
        }
    }
    return xml_node();
}

xml_attribute xml_node::attribute(const char* name) const
{
    if (!node_)
    {
        return xml_attribute();
    }
    for (const attr_record& a : node_->attributes)
    {
        if (a.name == name)
        {
            return xml_attribute(node_, &a);
        }
    }
    return xml_attribute();
}

xml_attribute xml_node::first_attribute() const
{
    return (node_ && !node_->attributes.empty()) ? xml_attribute(node_, &node_->attributes.front())
                                                 : xml_attribute();
}

xml_attribute xml_node::last_attribute() const
{
    return (node_ && !node_->attributes.empty()) ? xml_attribute(node_, &node_->attributes.back())
                                                 : xml_attribute();
}

const char* xml_node::child_value() const
{
    for (const node_record* c = node_ ? node_->first_child : nullptr; c; c = c->next_sibling)
    {
        if (c->type == node_pcdata || c->type == node_cdata)
        {
            return c->value.c_str();
        }
    }
    return "";
}

const char* xml_node::child_value(const char* name) const
{
    return child(name).child_value();
}

xml_object_range<xml_node_iterator> xml_node::children() const
{
    return xml_object_range<xml_node_iterator>(begin(), end());
}

xml_object_range<xml_named_node_iterator> xml_node::children(const char* name) const
{
    return xml_object_range<xml_named_node_iterator>(xml_named_node_iterator(child(name), name),
                                                     xml_named_node_iterator(xml_node(), name));
}

xml_object_range<xml_attribute_iterator> xml_node::attributes() const
{
    return xml_object_range<xml_attribute_iterator>(xml_attribute_iterator(first_attribute()),
                                                    xml_attribute_iterator());
}

xml_node_iterator xml_node::begin() const
{
    return xml_node_iterator(first_child());
}

xml_node_iterator xml_node::end() const
{
    return xml_node_iterator();
}

// ---------------------------------------------------------- xml_parse_result

const char* xml_parse_result::description() const
{
    switch (status)
    {
    case status_ok: return "No error";
    case status_file_not_found: return "File was not found";
    case status_io_error: return "Error reading from file";
    case status_out_of_memory: return "Could not allocate memory";
    case status_internal_error: return "Internal error";
    case status_unrecognized_tag: return "Could not determine tag type";
    case status_bad_pi: return "Unterminated document declaration or processing instruction";
    case status_bad_comment: return "Unterminated comment";
    case status_bad_cdata: return "Unterminated CDATA section";
    case status_bad_doctype: return "Unterminated document type declaration";
    case status_bad_pcdata: return "Malformed character data";
    case status_bad_start_element: return "Malformed start tag";
    case status_bad_attribute: return "Malformed attribute";
    case status_bad_end_element: return "Malformed end tag";
    case status_end_element_mismatch: return "Start and end tags do not match";
    case status_append_invalid_root: return "Nodes can only be appended to an element or a document";
    case status_no_document_element: return "No root element found";
    }
    return "Unknown error";
}

// ------------------------------------------------------------- xml_document

xml_document::xml_document()
{
    reset();
}

void xml_document::reset()
{
    nodes_.clear();
    nodes_.emplace_back();
    nodes_.front().type = node_document;
    node_ = &nodes_.front();
}

xml_node xml_document::document_element() const
{
    for (const node_record* c = nodes_.front().first_child; c; c = c->next_sibling)
    {
        if (c->type == node_element)
        {
            return xml_node(c);
        }
    }
    return xml_node();
}

xml_parse_result xml_document::load_buffer(const void* contents, std::size_t size, unsigned int, xml_encoding)
{
    reset();
    try
    {
        return Parser(nodes_, static_cast<const char*>(contents), size).Run();
    }
    catch (const std::bad_alloc&)
    {
        xml_parse_result r;
        r.status = status_out_of_memory;
        return r;
    }
}

xml_parse_result xml_document::load_string(const char* contents, unsigned int options)
{
    return load_buffer(contents, std::strlen(contents), options);
}

xml_parse_result xml_document::load_file(const char* path, unsigned int options, xml_encoding encoding)
{
    reset();
    xml_parse_result r;
    FILE* f = std::fopen(path, "rb");
    if (!f)
    {
        r.status = status_file_not_found;
        return r;
    }
    std::string data;
    char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0)
    {
        data.append(buf, n);
    }
    bool failed = std::ferror(f) != 0;
    std::fclose(f);
    if (failed)
    {
        r.status = status_io_error;
        return r;
    }
    return load_buffer(data.data(), data.size(), options, encoding);
}

} // namespace pugi
