// Prints the node stream that include/az_xmlreader.h reports for a file, one
// node per line: type, name, has-value, value, then the values of the
// attributes named on the command line ("-" where absent).  The last line is
// "end <result of the final xmlTextReaderRead>".  Built and run by
// tests/test_xml_reader.py.
#include <stdio.h>
#include <string>

#include "az_xmlreader.h"

static std::string Escape(const char *s) {
    std::string out;
    for (; s && *s; s++) {
        if (*s == '\n') out += "\\n";
        else if (*s == '\t') out += "\\t";
        else if (*s == '\\') out += "\\\\";
        else out += *s;
    }
    return out;
}

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    xmlTextReaderPtr r = xmlReaderForFile(argv[1], nullptr, XML_PARSE_NONET | XML_PARSE_HUGE);
    if (!r) {
        printf("open failed\n");
        return 1;
    }
    int rc;
    while ((rc = xmlTextReaderRead(r)) == 1) {
        const xmlChar *name = xmlTextReaderConstName(r);
        const xmlChar *value = xmlTextReaderConstValue(r);
        printf("%d\t%s\t%d\t%s", xmlTextReaderNodeType(r), name ? (const char *)name : "", xmlTextReaderHasValue(r),
               value ? Escape((const char *)value).c_str() : "-");
        for (int i = 2; i < argc; i++) {
            xmlChar *a = xmlTextReaderGetAttribute(r, (const xmlChar *)argv[i]);
            printf("\t%s", a ? Escape((const char *)a).c_str() : "-");
            if (a) xmlFree(a);
        }
        printf("\n");
    }
    printf("end %d\n", rc);
    xmlFreeTextReader(r);
    return 0;
}
