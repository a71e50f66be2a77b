/*
 * az_xmlreader.h -- the part of libxml2's streaming text reader that azimuth's
 * scene importer uses, header-only, for builds without libxml2.
 *
 * azimuth's ImportXML (src/azimuth_xml.cpp:3021-3930, through
 * src/azimuth_xml.h:6, `#include "libxml/xmlreader.h"`) walks a scene file
 * with xmlReaderForFile, xmlTextReaderRead, xmlTextReaderNodeType,
 * xmlTextReaderConstName, xmlTextReaderConstValue, xmlTextReaderHasValue,
 * xmlTextReaderGetAttribute, xmlFree and xmlFreeTextReader.  To build azimuth
 * (and import its XML scenes, PLY meshes included) where libxml2 is not
 * installed, put a file libxml/xmlreader.h on the include path that includes
 * this header.
 *
 * What it reads: elements with attributes (single or double quotes), empty
 * elements `<a/>`, text, comments, the XML declaration and processing
 * instructions (skipped), CDATA sections, a DOCTYPE without an
 * internal subset (skipped), the five predefined entities and character
 * references.  It reports nodes as libxml2's reader does with default
 * options: an element, then its children, then its end element (none for an
 * empty element); text that is all blanks is a significant-whitespace node
 * (type 14), other text a text node (3), a CDATA section a node of type 4.
 * Not supported: namespaces as such (prefixes stay part of the name), DTD
 * validation, external entities, encodings other than UTF-8/ASCII.  A
 * malformed file makes xmlTextReaderRead return -1.
 */
#ifndef AZ_XMLREADER_H
#define AZ_XMLREADER_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <utility>
#include <vector>

typedef unsigned char xmlChar;

#define LIBXML_READER_ENABLED 1
#define LIBXML_TEST_VERSION
#define XML_PARSE_NONET (1 << 11)
#define XML_PARSE_HUGE (1 << 19)

enum {
    AZ_XML_NODE_ELEMENT = 1,
    AZ_XML_NODE_TEXT = 3,
    AZ_XML_NODE_CDATA = 4,
    AZ_XML_NODE_COMMENT = 8,
    AZ_XML_NODE_SIGNIFICANT_WHITESPACE = 14,
    AZ_XML_NODE_END_ELEMENT = 15
};

struct az_xml_reader {
    std::string doc;                       // the whole file
    size_t pos = 0;
    bool failed = false;
    // the current node
    int type = 0;
    bool empty = false;                    // an element written <a/>
    std::string name, value;
    std::vector<std::pair<std::string, std::string>> attrs;
    std::vector<std::string> open;         // names of the open elements
    bool pending_end = false;              // an empty element still to be closed on the stack
    bool started = false;
};
typedef az_xml_reader *xmlTextReaderPtr;

static inline bool az_xml_is_blank(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }

static inline bool az_xml_name_char(char c) {
    return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_' || c == '-' ||
           c == '.' || c == ':' || (unsigned char)c >= 0x80;
}

// Appends the UTF-8 encoding of code point cp.
static inline void az_xml_put_utf8(std::string &out, unsigned long cp) {
    if (cp < 0x80) {
        out += (char)cp;
    } else if (cp < 0x800) {
        out += (char)(0xC0 | (cp >> 6));
        out += (char)(0x80 | (cp & 0x3F));
    } else if (cp < 0x10000) {
        out += (char)(0xE0 | (cp >> 12));
        out += (char)(0x80 | ((cp >> 6) & 0x3F));
        out += (char)(0x80 | (cp & 0x3F));
    } else {
        out += (char)(0xF0 | (cp >> 18));
        out += (char)(0x80 | ((cp >> 12) & 0x3F));
        out += (char)(0x80 | ((cp >> 6) & 0x3F));
        out += (char)(0x80 | (cp & 0x3F));
    }
}

// Replaces entity and character references; false on an unknown entity.
static inline bool az_xml_decode(const std::string &in, std::string &out) {
    out.clear();
    for (size_t i = 0; i < in.size(); i++) {
        if (in[i] != '&') {
            out += in[i];
            continue;
        }
        const size_t semi = in.find(';', i);
        if (semi == std::string::npos) return false;
        const std::string ent = in.substr(i + 1, semi - i - 1);
        if (ent == "lt") out += '<';
        else if (ent == "gt") out += '>';
        else if (ent == "amp") out += '&';
        else if (ent == "quot") out += '"';
        else if (ent == "apos") out += '\'';
        else if (ent.size() > 1 && ent[0] == '#') {
            char *end = nullptr;
            const unsigned long cp = ent[1] == 'x' ? strtoul(ent.c_str() + 2, &end, 16) : strtoul(ent.c_str() + 1, &end, 10);
            if (!end || *end != '\0' || cp == 0 || cp > 0x10FFFF) return false;
            az_xml_put_utf8(out, cp);
        } else {
            return false;
        }
        i = semi;
    }
    return true;
}

static inline xmlTextReaderPtr xmlReaderForFile(const char *path, const char *encoding, int options) {
    (void)encoding;
    (void)options;
    FILE *f = path ? fopen(path, "rb") : nullptr;
    if (!f) return nullptr;
    az_xml_reader *r = new az_xml_reader();
    char buf[65536];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) r->doc.append(buf, n);
    fclose(f);
    if (r->doc.size() >= 3 && (unsigned char)r->doc[0] == 0xEF && (unsigned char)r->doc[1] == 0xBB &&
        (unsigned char)r->doc[2] == 0xBF)
        r->pos = 3;   // UTF-8 byte order mark
    return r;
}

static inline void xmlFreeTextReader(xmlTextReaderPtr r) { delete r; }

// Advances to the next node: 1, 0 at the end of the document, -1 on an error.
static inline int xmlTextReaderRead(xmlTextReaderPtr r) {
    if (!r || r->failed) return -1;
    if (r->pending_end) {   // the element just reported was empty: it closes without an end node
        r->pending_end = false;
        r->open.pop_back();
    }
    const std::string &d = r->doc;
    for (;;) {
        r->attrs.clear();
        r->empty = false;
        if (r->pos >= d.size()) {
            if (!r->open.empty()) {
                r->failed = true;
                return -1;
            }
            return 0;
        }
        if (d[r->pos] != '<') {
            // character data up to the next markup
            const size_t lt = d.find('<', r->pos);
            const std::string raw = d.substr(r->pos, (lt == std::string::npos ? d.size() : lt) - r->pos);
            r->pos = lt == std::string::npos ? d.size() : lt;
            bool blank = true;
            for (char c : raw) blank = blank && az_xml_is_blank(c);
            if (r->open.empty()) {
                if (blank) continue;   // blanks around the root element are not nodes
                r->failed = true;
                return -1;
            }
            if (!az_xml_decode(raw, r->value)) {
                r->failed = true;
                return -1;
            }
            r->type = blank ? AZ_XML_NODE_SIGNIFICANT_WHITESPACE : AZ_XML_NODE_TEXT;
            r->name = "#text";
            return 1;
        }
        if (d.compare(r->pos, 4, "<!--") == 0) {
            const size_t e = d.find("-->", r->pos + 4);
            if (e == std::string::npos) {
                r->failed = true;
                return -1;
            }
            r->value = d.substr(r->pos + 4, e - r->pos - 4);
            r->pos = e + 3;
            r->type = AZ_XML_NODE_COMMENT;
            r->name = "#comment";
            return 1;
        }
        if (d.compare(r->pos, 9, "<![CDATA[") == 0) {
            const size_t e = d.find("]]>", r->pos + 9);
            if (e == std::string::npos || r->open.empty()) {
                r->failed = true;
                return -1;
            }
            r->value = d.substr(r->pos + 9, e - r->pos - 9);
            r->pos = e + 3;
            r->type = AZ_XML_NODE_CDATA;
            r->name = "#cdata-section";
            return 1;
        }
        if (d.compare(r->pos, 2, "<?") == 0) {   // XML declaration, processing instruction
            const size_t e = d.find("?>", r->pos + 2);
            if (e == std::string::npos) {
                r->failed = true;
                return -1;
            }
            r->pos = e + 2;
            continue;
        }
        if (d.compare(r->pos, 2, "<!") == 0) {   // DOCTYPE without an internal subset
            const size_t e = d.find('>', r->pos + 2);
            const size_t sub = d.find('[', r->pos + 2);
            if (e == std::string::npos || (sub != std::string::npos && sub < e)) {
                r->failed = true;
                return -1;
            }
            r->pos = e + 1;
            continue;
        }
        size_t p = r->pos + 1;
        const bool closing = p < d.size() && d[p] == '/';
        if (closing) p++;
        const size_t name_start = p;
        while (p < d.size() && az_xml_name_char(d[p])) p++;
        if (p == name_start) {
            r->failed = true;
            return -1;
        }
        r->name = d.substr(name_start, p - name_start);
        if (closing) {
            while (p < d.size() && az_xml_is_blank(d[p])) p++;
            if (p >= d.size() || d[p] != '>' || r->open.empty() || r->open.back() != r->name) {
                r->failed = true;
                return -1;
            }
            r->pos = p + 1;
            r->open.pop_back();
            r->type = AZ_XML_NODE_END_ELEMENT;
            r->value.clear();
            return 1;
        }
        // attributes
        for (;;) {
            while (p < d.size() && az_xml_is_blank(d[p])) p++;
            if (p >= d.size()) {
                r->failed = true;
                return -1;
            }
            if (d[p] == '>') {
                p++;
                break;
            }
            if (d[p] == '/' && p + 1 < d.size() && d[p + 1] == '>') {
                r->empty = true;
                p += 2;
                break;
            }
            const size_t an = p;
            while (p < d.size() && az_xml_name_char(d[p])) p++;
            if (p == an) {
                r->failed = true;
                return -1;
            }
            std::string aname = d.substr(an, p - an);
            while (p < d.size() && az_xml_is_blank(d[p])) p++;
            if (p >= d.size() || d[p] != '=') {
                r->failed = true;
                return -1;
            }
            p++;
            while (p < d.size() && az_xml_is_blank(d[p])) p++;
            if (p >= d.size() || (d[p] != '"' && d[p] != '\'')) {
                r->failed = true;
                return -1;
            }
            const char q = d[p++];
            const size_t ve = d.find(q, p);
            if (ve == std::string::npos) {
                r->failed = true;
                return -1;
            }
            std::string raw = d.substr(p, ve - p), val;
            if (raw.find('<') != std::string::npos) {   // not allowed unescaped in an attribute value
                r->failed = true;
                return -1;
            }
            for (char &c : raw)
                if (c == '\t' || c == '\n' || c == '\r') c = ' ';   // attribute-value normalisation
            if (!az_xml_decode(raw, val)) {
                r->failed = true;
                return -1;
            }
            r->attrs.emplace_back(std::move(aname), std::move(val));
            p = ve + 1;
        }
        r->pos = p;
        r->open.push_back(r->name);
        r->pending_end = r->empty;
        r->type = AZ_XML_NODE_ELEMENT;
        r->value.clear();
        r->started = true;
        return 1;
    }
}

static inline int xmlTextReaderNodeType(xmlTextReaderPtr r) { return r ? r->type : -1; }

static inline const xmlChar *xmlTextReaderConstName(xmlTextReaderPtr r) {
    return r && r->type ? (const xmlChar *)r->name.c_str() : nullptr;
}

static inline const xmlChar *xmlTextReaderConstValue(xmlTextReaderPtr r) {
    if (!r || r->type == AZ_XML_NODE_ELEMENT || r->type == AZ_XML_NODE_END_ELEMENT || r->type == 0) return nullptr;
    return (const xmlChar *)r->value.c_str();
}

static inline int xmlTextReaderHasValue(xmlTextReaderPtr r) {
    return r && (r->type == AZ_XML_NODE_TEXT || r->type == AZ_XML_NODE_CDATA ||
                 r->type == AZ_XML_NODE_COMMENT || r->type == AZ_XML_NODE_SIGNIFICANT_WHITESPACE);
}

// A copy of the named attribute of the current element (free with xmlFree), or null.
static inline xmlChar *xmlTextReaderGetAttribute(xmlTextReaderPtr r, const xmlChar *name) {
    if (!r || !name || r->type != AZ_XML_NODE_ELEMENT) return nullptr;
    for (const auto &a : r->attrs)
        if (a.first == (const char *)name) {
            char *s = (char *)malloc(a.second.size() + 1);
            if (s) memcpy(s, a.second.c_str(), a.second.size() + 1);
            return (xmlChar *)s;
        }
    return nullptr;
}

static inline void az_xml_free(void *p) { free(p); }
#define xmlFree az_xml_free

#endif
