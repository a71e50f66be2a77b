/* Oracle-build stub for the libxml2 text reader (no libxml2 in this image).
 * xmlReaderForFile always fails, so ImportXML returns failure cleanly; the
 * oracle builds its scenes in memory instead.                              */
#pragma once
#include <stdlib.h>
typedef unsigned char xmlChar;
typedef struct az_xml_reader_stub *xmlTextReaderPtr;
static inline xmlTextReaderPtr xmlReaderForFile(const char *, const char *, int) { return 0; }
static inline int xmlTextReaderRead(xmlTextReaderPtr) { return -1; }
static inline int xmlTextReaderNodeType(xmlTextReaderPtr) { return -1; }
static inline int xmlTextReaderHasValue(xmlTextReaderPtr) { return 0; }
static inline const xmlChar *xmlTextReaderConstName(xmlTextReaderPtr) { return 0; }
static inline const xmlChar *xmlTextReaderConstValue(xmlTextReaderPtr) { return 0; }
static inline xmlChar *xmlTextReaderGetAttribute(xmlTextReaderPtr, const xmlChar *) { return 0; }
static inline void xmlFreeTextReader(xmlTextReaderPtr) {}
static inline void az_xml_free_stub(void *p) { free(p); }
#define xmlFree az_xml_free_stub
