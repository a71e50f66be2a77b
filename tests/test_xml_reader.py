"""The header-only text reader (include/az_xmlreader.h) that stands in for
libxml2's xmlTextReader under azimuth's ImportXML (src/azimuth_xml.h:6,
src/azimuth_xml.cpp:3021-3930).  The node stream it reports must be the one
libxml2's reader reports with default options, as the importer's loop
(src/azimuth_xml.cpp:3136-3227) reads it: element, children, end element (no
end element for <a/>), blank text as significant whitespace (14), other text
as text (3), CDATA as its own type (4), comments (8); -1 on malformed input.
Runs tests/xml_walk.cpp, compiled against the header."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")


@pytest.fixture(scope="module")
def walker(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("xmlwalk") / "xml_walk")
    subprocess.run(["g++", "-std=c++14", "-O1", "-Wall", "-Werror", "-I", INCLUDE,
                    os.path.join(HERE, "xml_walk.cpp"), "-o", out], check=True)
    return out


def walk(walker, tmp_path, text, attrs=(), raw=False):
    p = tmp_path / "in.xml"
    p.write_bytes(text if raw else text.encode())
    res = subprocess.run([walker, str(p)] + list(attrs), capture_output=True, text=True, check=True)
    lines = res.stdout.splitlines()
    assert lines[-1].startswith("end ")
    nodes = [tuple(int(f) if i in (0, 2) else f for i, f in enumerate(l.split("\t"))) for l in lines[:-1]]
    return nodes, int(lines[-1][4:])


def test_node_stream_follows_libxml2(walker, tmp_path):
    text = ('<?xml version="1.0" encoding="UTF-8"?>\n<!-- c -->\n<Scene a="1" b=\'two\'>\n'
            '  <X>1 2 3</X>\n  <Faces plyFile="f.ply"/>\n  <E></E>\n</Scene>\n')
    nodes, rc = walk(walker, tmp_path, text, ["a", "b", "plyFile"])
    ws = "\\n  "
    assert nodes == [
        (8, "#comment", 1, " c ", "-", "-", "-"),
        (1, "Scene", 0, "-", "1", "two", "-"),
        (14, "#text", 1, ws, "-", "-", "-"),
        (1, "X", 0, "-", "-", "-", "-"),
        (3, "#text", 1, "1 2 3", "-", "-", "-"),
        (15, "X", 0, "-", "-", "-", "-"),
        (14, "#text", 1, ws, "-", "-", "-"),
        (1, "Faces", 0, "-", "-", "-", "f.ply"),     # empty element: no end element follows
        (14, "#text", 1, ws, "-", "-", "-"),
        (1, "E", 0, "-", "-", "-", "-"),
        (15, "E", 0, "-", "-", "-", "-"),
        (14, "#text", 1, "\\n", "-", "-", "-"),
        (15, "Scene", 0, "-", "-", "-", "-"),
    ]
    assert rc == 0


def test_references_cdata_and_attribute_blanks(walker, tmp_path):
    text = ('<a t="x &amp; y &#65;&#x42;" n="l1\nl2\tz">&lt;b&gt; &quot;q&quot; &apos;&#xe9;'
            '<c/><![CDATA[1 <2> &amp;]]></a>')
    nodes, rc = walk(walker, tmp_path, text, ["t", "n"])
    assert nodes == [
        (1, "a", 0, "-", "x & y AB", "l1 l2 z"),
        (3, "#text", 1, "<b> \"q\" 'é", "-", "-"),
        (1, "c", 0, "-", "-", "-"),
        (4, "#cdata-section", 1, "1 <2> &amp;", "-", "-"),
        (15, "a", 0, "-", "-", "-"),
    ]
    assert rc == 0


def test_prolog_forms_are_skipped(walker, tmp_path):
    text = b'\xef\xbb\xbf<?xml version="1.0"?>\n<!DOCTYPE Scene SYSTEM "s.dtd">\n<?pi x?>\n<Scene/>\n'
    nodes, rc = walk(walker, tmp_path, text, raw=True)
    assert nodes == [(1, "Scene", 0, "-")] and rc == 0


@pytest.mark.parametrize("text", [
    "<a><b></a>",                 # mismatched end tag
    "<a><b/>",                    # element never closed
    "<a>x &nbsp; y</a>",          # entity that is not predefined
    "text<a/>",                   # character data outside the root element
    "<a b=1/>",                   # unquoted attribute value
    "<a><!-- open comment</a>",   # comment never closed
    "<a>&#0;</a>",                # character reference to NUL
    "<a b='<c/>'/>",              # '<' inside an attribute value
])
def test_malformed_input_is_an_error(walker, tmp_path, text):
    _, rc = walk(walker, tmp_path, text)
    assert rc == -1


def test_missing_file_gives_no_reader(walker, tmp_path):
    res = subprocess.run([walker, str(tmp_path / "absent.xml")], capture_output=True, text=True)
    assert res.returncode == 1 and "open failed" in res.stdout


def test_markup_inside_values_and_nesting(walker, tmp_path):
    text = ('<a k = "x>y" j=\'z/\'><a><!--c--><b/></a>t<a/></a>')
    nodes, rc = walk(walker, tmp_path, text, ["k", "j"])
    assert nodes == [
        (1, "a", 0, "-", "x>y", "z/"),
        (1, "a", 0, "-", "-", "-"),
        (8, "#comment", 1, "c", "-", "-"),
        (1, "b", 0, "-", "-", "-"),
        (15, "a", 0, "-", "-", "-"),
        (3, "#text", 1, "t", "-", "-"),
        (1, "a", 0, "-", "-", "-"),
        (15, "a", 0, "-", "-", "-"),
    ]
    assert rc == 0
