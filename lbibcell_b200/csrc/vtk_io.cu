// vtk_io.cu — VTK XML (ASCII) reading and writing without VTK.  Host code.
//
// Reader: Geometry::loadGeometryVTK (Geometry.cpp:162-306).  Of the blocks
// listed in the .vtm, exactly one must be poly data with polygons; its points
// become GeometryNodes 0..n-1 (a Float32 point array is read as float, as
// vtkPoints stores it, then widened), and each polygon i1..in becomes the
// connections (i1,i2) .. (i(n-1),in) and the closing (in,i1), with the domain
// and cell type of the polygon's first point and, for connection (ik, ik+1),
// the boundary descriptor string of point ik (the closing connection reuses
// the last one parsed, as the reference's loop variable does).
//
// Writers: the blocks of vtkCellReporter, vtkForceReporter, vtkCDEReporter
// and vtkFluidReporter, appended to <prefix>_<time>.vtm as those functors do.
#include "vtk_io.h"

#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace lbib {
namespace vtk {

namespace {

std::string slurp(const std::string& path, const char* missing) {
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) throw std::runtime_error(missing);
    std::stringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

std::string dir_of(const std::string& path) {
    const size_t p = path.find_last_of('/');
    return p == std::string::npos ? std::string() : path.substr(0, p + 1);
}

std::string stem_of(const std::string& path) {
    const size_t p = path.find_last_of('/');
    std::string f = p == std::string::npos ? path : path.substr(p + 1);
    if (f.size() > 4 && f.compare(f.size() - 4, 4, ".vtm") == 0) f.resize(f.size() - 4);
    return f;
}

// Value of attribute `name` in the start tag `tag` ("" when absent).
std::string attr(const std::string& tag, const std::string& name) {
    const std::string key = " " + name + "=\"";
    const size_t p = tag.find(key);
    if (p == std::string::npos) return std::string();
    const size_t b = p + key.size();
    const size_t e = tag.find('"', b);
    return e == std::string::npos ? std::string() : tag.substr(b, e - b);
}

// An element <name ...>content</name> found in s[from, to).
struct Elem {
    std::string tag;       // the start tag
    size_t begin = 0;      // content
    size_t end = 0;
    size_t after = 0;      // past the end tag
    bool found = false;
};

Elem find_elem(const std::string& s, size_t from, size_t to, const std::string& name,
               const std::string& attrName = std::string(), const std::string& attrValue = std::string()) {
    Elem e;
    const std::string open = "<" + name;
    size_t p = from;
    while (true) {
        p = s.find(open, p);
        if (p == std::string::npos || p >= to) return e;
        const char c = s[p + open.size()];
        if (c != ' ' && c != '>' && c != '/' && c != '\t' && c != '\n' && c != '\r') {
            p += open.size();
            continue;
        }
        const size_t te = s.find('>', p);
        if (te == std::string::npos) return e;
        const std::string tag = s.substr(p, te - p + 1);
        if (!attrName.empty() && attr(tag, attrName) != attrValue) {
            p = te;
            continue;
        }
        e.tag = tag;
        if (tag[tag.size() - 2] == '/') {  // empty element
            e.begin = e.end = te + 1;
            e.after = te + 1;
        } else {
            const std::string close = "</" + name + ">";
            const size_t ce = s.find(close, te);
            if (ce == std::string::npos) return e;
            e.begin = te + 1;
            e.end = ce;
            e.after = ce + close.size();
        }
        e.found = true;
        return e;
    }
}

void require_ascii(const Elem& e, const std::string& file) {
    const std::string f = attr(e.tag, "format");
    if (f != "ascii")
        throw std::runtime_error("VTK file " + file + ": array " + attr(e.tag, "Name") + " is not in ascii format");
}

std::vector<double> parse_doubles(const std::string& s, const Elem& e, bool asFloat) {
    std::vector<double> v;
    const char* p = s.c_str() + e.begin;
    const char* end = s.c_str() + e.end;
    while (p < end) {
        char* q = nullptr;
        double d;
        if (asFloat) d = (double)std::strtof(p, &q);
        else d = std::strtod(p, &q);
        if (q == p) {
            ++p;
            continue;
        }
        if (q > end) break;
        v.push_back(d);
        p = q;
    }
    return v;
}

std::vector<long long> parse_ints(const std::string& s, const Elem& e) {
    std::vector<long long> v;
    const char* p = s.c_str() + e.begin;
    const char* end = s.c_str() + e.end;
    while (p < end) {
        char* q = nullptr;
        const long long d = std::strtoll(p, &q, 10);
        if (q == p) {
            ++p;
            continue;
        }
        if (q > end) break;
        v.push_back(d);
        p = q;
    }
    return v;
}

// A vtkStringArray in ASCII: the character codes of each string, then 0.
std::vector<std::string> parse_strings(const std::string& s, const Elem& e) {
    std::vector<std::string> out;
    std::string cur;
    for (long long c : parse_ints(s, e)) {
        if (c == 0) {
            out.push_back(cur);
            cur.clear();
        } else {
            cur.push_back((char)c);
        }
    }
    return out;
}

// "bs cde bs cde ..." into the reference's map<string, vector<string>>, back
// into this library's descriptor string.
std::string descriptor(const std::string& text) {
    std::stringstream ls(text);
    std::map<std::string, std::vector<std::string>> type;
    std::string a, b;
    while (ls >> a >> b) type[a].push_back(b);
    std::string d;
    for (const auto& kv : type)
        for (const auto& c : kv.second) d += "\t" + kv.first + "\t" + c;
    return d;
}

}  // namespace

void read_vtm_geometry(const std::string& path, Geometry& g) {
    struct stat st;
    if (stat(path.c_str(), &st) != 0) throw std::runtime_error("Cannot find the geometry.vtm file.");
    const std::string vtm = slurp(path, "Cannot find the geometry.vtm file.");
    const std::string dir = dir_of(path);
    // the blocks, in order; candidates are poly data with polygons
    std::string polyFile, polyText;
    int candidates = 0;
    size_t p = 0;
    while (true) {
        const Elem ds = find_elem(vtm, p, vtm.size(), "DataSet");
        if (!ds.found) break;
        p = ds.after;
        const std::string file = attr(ds.tag, "file");
        if (file.empty()) continue;
        const std::string text = slurp(dir + file, "Cannot open a block file of the geometry.vtm file.");
        const Elem vf = find_elem(text, 0, text.size(), "VTKFile");
        if (!vf.found || attr(vf.tag, "type") != "PolyData") continue;
        const Elem piece = find_elem(text, 0, text.size(), "Piece");
        if (!piece.found || std::atol(attr(piece.tag, "NumberOfPolys").c_str()) <= 0) continue;
        ++candidates;
        polyFile = dir + file;
        polyText = text;
    }
    if (candidates != 1)
        throw std::runtime_error("more or less than one vtk polygon block found in input geometry file found.");
    const std::string& s = polyText;
    const Elem piece = find_elem(s, 0, s.size(), "Piece");
    // points
    const Elem pts = find_elem(s, piece.begin, piece.end, "Points");
    const Elem pa = find_elem(s, pts.begin, pts.end, "DataArray");
    if (!pts.found || !pa.found) throw std::runtime_error("no points in " + polyFile);
    require_ascii(pa, polyFile);
    const int nc = attr(pa.tag, "NumberOfComponents").empty() ? 1 : std::atoi(attr(pa.tag, "NumberOfComponents").c_str());
    if (nc != 3) throw std::runtime_error("points of " + polyFile + " do not have 3 components");
    const std::vector<double> xyz = parse_doubles(s, pa, attr(pa.tag, "type") == "Float32");
    const size_t n = xyz.size() / 3;
    g.x.resize(n);
    g.y.resize(n);
    for (size_t k = 0; k < n; ++k) {
        g.x[k] = xyz[3 * k];
        g.y[k] = xyz[3 * k + 1];
    }
    // point attributes
    const Elem pd = find_elem(s, piece.begin, piece.end, "PointData");
    const Elem dArr = find_elem(s, pd.begin, pd.end, "DataArray", "Name", "domain_identifier");
    if (!pd.found || !dArr.found) throw std::runtime_error("domain_identifier array not found in vtk input file.");
    const Elem cArr = find_elem(s, pd.begin, pd.end, "DataArray", "Name", "cell_type");
    if (!cArr.found) throw std::runtime_error("cell_type array not found in vtk input file.");
    Elem bArr = find_elem(s, pd.begin, pd.end, "Array", "Name", "boundarydescriptors");
    if (!bArr.found) throw std::runtime_error("boundarydescriptor array not found in vtk input file");
    require_ascii(dArr, polyFile);
    require_ascii(cArr, polyFile);
    require_ascii(bArr, polyFile);
    const std::vector<double> dom = parse_doubles(s, dArr, false);
    const std::vector<double> ctype = parse_doubles(s, cArr, false);
    const std::vector<std::string> bstr = parse_strings(s, bArr);
    if (dom.size() < n || ctype.size() < n || bstr.size() < n)
        throw std::runtime_error("point arrays of " + polyFile + " are shorter than the point list");
    // polygons
    const Elem polys = find_elem(s, piece.begin, piece.end, "Polys");
    const Elem con = find_elem(s, polys.begin, polys.end, "DataArray", "Name", "connectivity");
    const Elem off = find_elem(s, polys.begin, polys.end, "DataArray", "Name", "offsets");
    if (!polys.found || !con.found || !off.found) throw std::runtime_error("no polygons in " + polyFile);
    require_ascii(con, polyFile);
    require_ascii(off, polyFile);
    const std::vector<long long> ids = parse_ints(s, con);
    const std::vector<long long> offsets = parse_ints(s, off);
    g.cellType.clear();
    g.cellType[0] = 0;  // fluid default
    g.conns.clear();
    std::string last;  // the descriptor parsed last (survives polygons)
    long long b = 0;
    for (long long e : offsets) {
        if (e <= b || e > (long long)ids.size()) throw std::runtime_error("bad polygon offsets in " + polyFile);
        for (long long k = b; k < e; ++k)
            if (ids[k] < 0 || ids[k] >= (long long)n) throw std::runtime_error("bad point id in " + polyFile);
        const uint32_t d = (uint32_t)dom[ids[b]];
        g.cellType[d] = (uint32_t)ctype[ids[b]];
        for (long long k = b; k + 1 < e; ++k) {
            last = descriptor(bstr[ids[k]]);
            g.conns.push_back(Conn{(uint32_t)ids[k], (uint32_t)ids[k + 1], d, last});
        }
        g.conns.push_back(Conn{(uint32_t)ids[e - 1], (uint32_t)ids[b], d, last});
        b = e;
    }
}

// ---------------------------------------------------------------------------
// Writers

namespace {

std::string num(double v, const std::string& type) {
    char buf[40];
    if (type == "Float32") std::snprintf(buf, sizeof buf, "%.9g", (double)(float)v);
    else if (type == "Float64") std::snprintf(buf, sizeof buf, "%.17g", v);
    else std::snprintf(buf, sizeof buf, "%lld", (long long)v);
    return buf;
}

// Range attributes as VTK writes them: the value range of a one-component
// array, the range of the tuple norms otherwise; an empty array gets
// 1e+299 / -1e+299.
std::string range_attrs(const std::vector<double>& v, int comps, const std::string& type) {
    if (v.empty()) return " RangeMin=\"1e+299\" RangeMax=\"-1e+299\"";
    double lo = INFINITY, hi = -INFINITY;
    for (size_t t = 0; t + comps <= v.size(); t += comps) {
        double x = 0;
        if (comps == 1) {
            x = v[t];
        } else {
            for (int c = 0; c < comps; ++c) {
                const double w = type == "Float32" ? (double)(float)v[t + c] : v[t + c];
                x += w * w;
            }
            x = std::sqrt(x);
        }
        lo = std::min(lo, x);
        hi = std::max(hi, x);
    }
    const std::string t = comps == 1 ? type : std::string("Float64");
    return " RangeMin=\"" + num(lo, t) + "\" RangeMax=\"" + num(hi, t) + "\"";
}

void write_values(std::ostream& o, const std::vector<double>& v, const std::string& type, const std::string& indent) {
    for (size_t k = 0; k < v.size(); ++k) {
        if (k % 6 == 0) o << (k ? "\n" : "") << indent;
        else o << ' ';
        o << num(v[k], type);
    }
    if (!v.empty()) o << "\n";
}

void write_array(std::ostream& o, const Array& a, const std::string& indent) {
    o << indent << "<DataArray type=\"" << a.type << "\" Name=\"" << a.name << "\"";
    if (a.components != 1) o << " NumberOfComponents=\"" << a.components << "\"";
    o << " format=\"ascii\"" << range_attrs(a.values, a.components, a.type) << ">\n";
    write_values(o, a.values, a.type, indent + "  ");
    o << indent << "</DataArray>\n";
}

void write_string_array(std::ostream& o, const std::string& name, const std::vector<std::string>& v,
                        const std::string& indent) {
    o << indent << "<Array type=\"String\" Name=\"" << name << "\" format=\"ascii\">\n";
    std::vector<double> codes;
    for (const auto& str : v) {
        for (unsigned char c : str) codes.push_back((double)c);
        codes.push_back(0.0);
    }
    write_values(o, codes, "UInt8", indent + "  ");
    o << indent << "</Array>\n";
}

void write_cells(std::ostream& o, const char* name, const std::vector<int64_t>* con, const std::vector<int64_t>* off) {
    const std::string in = "      ";
    o << in << "<" << name << ">\n";
    std::vector<double> c, f;
    if (con) c.assign(con->begin(), con->end());
    if (off) f.assign(off->begin(), off->end());
    write_array(o, Array{"connectivity", 1, "Int64", c}, in + "  ");
    write_array(o, Array{"offsets", 1, "Int64", f}, in + "  ");
    o << in << "</" << name << ">\n";
}

// The blocks already listed in the .vtm, in order.
std::vector<std::string> listed_blocks(const std::string& vtm) {
    std::vector<std::string> files;
    struct stat st;
    if (stat(vtm.c_str(), &st) != 0) return files;
    const std::string s = slurp(vtm, "cannot read the .vtm file");
    size_t p = 0;
    while (true) {
        const Elem ds = find_elem(s, p, s.size(), "DataSet");
        if (!ds.found) break;
        p = ds.after;
        files.push_back(attr(ds.tag, "file"));
    }
    return files;
}

// Writes the next block's file (text from `body`) and the .vtm listing it.
template <typename Body>
void append(const std::string& vtm, const char* ext, Body body) {
    std::vector<std::string> files = listed_blocks(vtm);
    const std::string stem = stem_of(vtm);
    const std::string dir = dir_of(vtm);
    const std::string sub = stem + "/" + stem + "_" + std::to_string(files.size()) + ext;
    mkdir((dir + stem).c_str(), 0755);
    {
        std::ofstream o(dir + sub);
        if (!o.is_open()) throw std::runtime_error("The output file could not be opened: " + dir + sub);
        o << "<?xml version=\"1.0\"?>\n";
        body(o);
        if (!o.good()) throw std::runtime_error("write failed: " + dir + sub);
    }
    files.push_back(sub);
    std::ofstream o(vtm);
    if (!o.is_open()) throw std::runtime_error("The output file could not be opened: " + vtm);
    o << "<?xml version=\"1.0\"?>\n"
      << "<VTKFile type=\"vtkMultiBlockDataSet\" version=\"1.0\" byte_order=\"LittleEndian\">\n"
      << "  <vtkMultiBlockDataSet>\n";
    for (size_t k = 0; k < files.size(); ++k)
        o << "    <DataSet index=\"" << k << "\" file=\"" << files[k] << "\">\n    </DataSet>\n";
    o << "  </vtkMultiBlockDataSet>\n</VTKFile>\n";
    if (!o.good()) throw std::runtime_error("write failed: " + vtm);
}

}  // namespace

void append_block(const std::string& vtm, const PolyData& pd) {
    append(vtm, ".vtp", [&](std::ostream& o) {
        const size_t np = pd.px.size(), nc = pd.offsets.size();
        o << "<VTKFile type=\"PolyData\" version=\"0.1\" byte_order=\"LittleEndian\">\n  <PolyData>\n"
          << "    <Piece NumberOfPoints=\"" << np << "\" NumberOfVerts=\"0\" NumberOfLines=\"" << (pd.lines ? nc : 0)
          << "\" NumberOfStrips=\"0\" NumberOfPolys=\"" << (pd.lines ? 0 : nc) << "\">\n";
        o << "      <PointData>\n";
        for (const auto& a : pd.pointData) write_array(o, a, "        ");
        for (const auto& sa : pd.pointStrings) write_string_array(o, sa.first, sa.second, "        ");
        o << "      </PointData>\n      <CellData>\n";
        for (const auto& a : pd.cellData) write_array(o, a, "        ");
        o << "      </CellData>\n      <Points>\n";
        Array pts{"Points", 3, "Float32", {}};
        pts.values.reserve(3 * np);
        for (size_t k = 0; k < np; ++k) {
            pts.values.push_back(pd.px[k]);
            pts.values.push_back(pd.py[k]);
            pts.values.push_back(0.0);
        }
        write_array(o, pts, "        ");
        o << "      </Points>\n";
        write_cells(o, "Verts", nullptr, nullptr);
        write_cells(o, "Lines", pd.lines ? &pd.connectivity : nullptr, pd.lines ? &pd.offsets : nullptr);
        write_cells(o, "Strips", nullptr, nullptr);
        write_cells(o, "Polys", pd.lines ? nullptr : &pd.connectivity, pd.lines ? nullptr : &pd.offsets);
        o << "    </Piece>\n  </PolyData>\n</VTKFile>\n";
    });
}

void append_block(const std::string& vtm, const ImageData& im) {
    append(vtm, ".vti", [&](std::ostream& o) {
        const std::string ext = "0 " + std::to_string(im.X - 1) + " 0 " + std::to_string(im.Y - 1) + " 0 0";
        const std::string sp = num(im.spacing, "Float64");
        o << "<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
          << "  <ImageData WholeExtent=\"" << ext << "\" Origin=\"0 0 0\" Spacing=\"" << sp << " " << sp << " " << sp
          << "\">\n  <Piece Extent=\"" << ext << "\">\n    <PointData>\n";
        for (const auto& a : im.pointData) write_array(o, a, "      ");
        o << "    </PointData>\n    <CellData>\n    </CellData>\n  </Piece>\n  </ImageData>\n</VTKFile>\n";
    });
}

}  // namespace vtk
}  // namespace lbib
