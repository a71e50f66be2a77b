/* libxml/xmlreader.h for the oracle build of azimuth (no libxml2 in this
 * image): the header-only text reader of include/az_xmlreader.h, so that
 * azimuth's own ImportXML (src/azimuth_xml.cpp:3021-3930) and its PLY loader
 * run unmodified.                                                          */
#pragma once
#include "az_xmlreader.h"
