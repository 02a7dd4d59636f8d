// Host engine: environment loading (reference file formats and validation),
// device residency, coefficient-tile construction and kernel launches.
#include <algorithm>
#include <atomic>
#include <array>
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <exception>
#include <functional>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <system_error>
#include <thread>

#include <cub/device/device_radix_sort.cuh>

#include "engine.hpp"

namespace phop {

static double mjdToEtHost(double mjd) { return std::fma(mjd, 86400.0, -43200.0); }
static double etToMjdHost(double et) { return std::fma(et, 1.0 / 86400.0, 0.5); }

#define PHOP_CUDA(call)                                                                                    \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_)); \
    } while (0)

// ---- naming (IF/naming/points/Registry.h, NAIF ids) ------------------------------------------------
static int naifId(const std::string& name) {
    static const std::map<std::string, int> ids = {
        {"Sun", 10}, {"Moon", 301}, {"Earth", 399}, {"MercuryBarycenter", 1}, {"VenusBarycenter", 2},
        {"EarthMoonBarycenter", 3}, {"MarsBarycenter", 4}, {"JupiterBarycenter", 5}, {"SaturnBarycenter", 6},
        {"UranusBarycenter", 7}, {"NeptuneBarycenter", 8}, {"PlutoBarycenter", 9}};
    auto it = ids.find(name);
    if (it == ids.end()) throw std::runtime_error("Unknown body name: " + name);
    return it->second;
}

// ---- loaders ------------------------------------------------------------------------------------------
// Lines of a text file, as std::getline(…, '\n') yields them.
class TextLines {
public:
    explicit TextLines(const std::string& text) : p_(text.data()), end_(text.data() + text.size()) {}
    bool next(const char*& b, const char*& e) {
        if (p_ >= end_) return false;
        const char* nl = (const char*)std::memchr(p_, '\n', (size_t)(end_ - p_));
        b = p_;
        e = nl ? nl : end_;
        p_ = nl ? nl + 1 : end_;
        return true;
    }

private:
    const char* p_;
    const char* end_;
};

// Whitespace-separated fields of one line, read as std::istream's >> reads an
// int or a double: after white space, the longest [sign]digits[.digits]
// [e[sign]digits] prefix (an exponent only after a mantissa digit), which
// must convert whole; an out-of-range int or an infinite double fails.
class LineFields {
public:
    LineFields(const char* b, const char* e) : p_(b), end_(e) {}
    bool readInt(int& v) {
        const char* s = start();
        if (p_ < end_ && (*p_ == '+' || *p_ == '-')) ++p_;
        const char* d = p_;
        digits();
        if (p_ == d) return false;
        errno = 0;
        const long long x = std::strtoll(copy(s), nullptr, 10);
        if (errno == ERANGE || x < INT32_MIN || x > INT32_MAX) return false;
        v = (int)x;
        return true;
    }
    bool readDouble(double& v) {
        const char* s = start();
        if (p_ < end_ && (*p_ == '+' || *p_ == '-')) ++p_;
        const char* m = p_;
        digits();
        bool mantissa = p_ != m;
        if (p_ < end_ && *p_ == '.') {
            ++p_;
            const char* f = p_;
            digits();
            mantissa = mantissa || p_ != f;
        }
        if (mantissa && p_ < end_ && (*p_ == 'e' || *p_ == 'E')) {
            ++p_;
            if (p_ < end_ && (*p_ == '+' || *p_ == '-')) ++p_;
            digits();
        }
        if (p_ == s) return false;
        char* stop = nullptr;
        const double x = std::strtod(copy(s), &stop);
        if (*stop != 0 || std::isinf(x)) return false;
        v = x;
        return true;
    }

private:
    const char* start() {
        while (p_ < end_ && std::isspace((unsigned char)*p_)) ++p_;
        return p_;
    }
    void digits() {
        while (p_ < end_ && *p_ >= '0' && *p_ <= '9') ++p_;
    }
    // the field [s, p_) as a C string
    const char* copy(const char* s) {
        field_.assign(s, (size_t)(p_ - s));
        return field_.c_str();
    }
    const char* p_;
    const char* end_;
    std::string field_;
};

static void loadConstants(const std::string& path, HostEnvironment& env) {
    const Value c = parseJson(readTextFile(path));
    if (!c.isArray()) throw std::runtime_error("Constants file must hold a JSON array: " + path);
    for (const Value& item : c.items()) {
        if (const Value* au = item.find("AU")) env.au = au->asDouble();
        if (const Value* id = item.find("NAIFID")) {
            const int nid = (int)id->asInt();
            if (const Value* gm = item.find("GM")) env.constGm[nid] = gm->asDouble();
            if (const Value* r = item.find("R")) env.constRadius[nid] = r->asDouble();
            // ConstantsJson.h:57-76: J2 defaults to 0, SOIOld takes precedence over SOI
            env.constJ2[nid] = item.find("J2") ? item.at("J2").asDouble() : 0.0;
            env.constSoi[nid] = item.find("SOIOld") ? item.at("SOIOld").asDouble()
                                                    : (item.find("SOI") ? item.at("SOI").asDouble() : 1e20);
        }
    }
    if (env.au <= 0) throw std::runtime_error("Constants file lacks AU: " + path);
}

// PDS-SHA table (Coefficients.h:241-362)
static void loadShTable(const Value& shape, HostEnvironment& env) {
    const std::string path = shape.at("file").asString();
    const std::string delimStr = shape.find("delimiter") ? shape.at("delimiter").asString() : std::string(",");
    const char delim = delimStr.empty() ? ',' : delimStr[0];
    const int headerLines = shape.find("headerLines") ? (int)shape.at("headerLines").asInt() : 0;
    const int reqDeg = shape.find("degree") ? (int)shape.at("degree").asInt() : -1;
    const int reqOrd = shape.find("order") ? (int)shape.at("order").asInt() : -1;
    const std::string text = readTextFile(path);
    TextLines lines(text);
    const char *lb, *le;
    std::vector<std::vector<double>> rows;
    std::string tok;
    int skip = headerLines;
    while (lines.next(lb, le)) {
        if (skip > 0) {
            --skip;
            continue;
        }
        // fields split at the delimiter, leading blanks dropped, blank fields skipped, read by std::stod
        std::vector<double> row;
        bool any = false;
        for (const char* q = lb; q < le;) {
            const char* te = (const char*)std::memchr(q, delim, (size_t)(le - q));
            if (!te) te = le;
            const char* a = q;
            while (a < te && (*a == ' ' || *a == '\t' || *a == '\r')) ++a;
            if (a < te) {
                tok.assign(a, (size_t)(te - a));
                row.push_back(std::stod(tok));
                any = true;
            }
            q = te < le ? te + 1 : le;
        }
        if (any) rows.push_back(std::move(row));
    }
    if (rows.empty()) throw std::runtime_error("No coefficients found in file: " + path);
    const auto& h = rows.front();
    if (h.size() != 8)
        throw std::runtime_error("Invalid PDS-SHA header in file: " + path + " - Expected 8 values, found "
                                 + std::to_string(h.size()));
    const int maxDegH = (int)h[3], maxOrdH = (int)h[4], norm = (int)h[5];
    if (reqDeg != -1 && reqDeg > maxDegH)
        throw std::runtime_error("Requested maximum degree " + std::to_string(reqDeg)
                                 + " exceeds available maximum degree " + std::to_string(maxDegH) + " in file: " + path);
    if (reqOrd != -1 && reqOrd > maxOrdH)
        throw std::runtime_error("Requested maximum order " + std::to_string(reqOrd)
                                 + " exceeds available maximum order " + std::to_string(maxOrdH) + " in file: " + path);
    if (norm != 0 && norm != 1) throw std::runtime_error("Unsupported normalization flag in file: " + path);
    if (h[6] != 0.0 || h[7] != 0.0) throw std::runtime_error("Non-zero latitude/longitude offsets are not supported.");
    env.shDegree = reqDeg == -1 ? maxDegH : reqDeg;
    env.shOrder = reqOrd == -1 ? maxOrdH : reqOrd;
    if (env.shOrder > env.shDegree) env.shOrder = env.shDegree;
    if (env.shDegree <= 0) throw std::runtime_error("Maximum degree must be > 0");
    env.shNormalized = norm;
    env.shR = h[0];
    env.shGM = h[1];
    const size_t tri = (size_t)(env.shDegree + 1) * (env.shDegree + 2) / 2;
    env.shC.assign(tri, 0.0);
    env.shS.assign(tri, 0.0);
    for (size_t i = 1; i < rows.size(); ++i) {
        const auto& r = rows[i];
        if (r.size() != 4 && r.size() != 6)
            throw std::runtime_error("Invalid coefficient row in file: " + path + " - Expected 6 values, found "
                                     + std::to_string(r.size()));
        const int n = (int)r[0], m = (int)r[1];
        if (n <= 0) throw std::runtime_error("Invalid degree 0 coefficient found in file: " + path);
        if (m > n) throw std::runtime_error("Invalid order " + std::to_string(m) + " for degree " + std::to_string(n)
                                            + " found in file: " + path);
        if (m == 0 && r[3] != 0.0) throw std::runtime_error("Invalid non-zero Sn0 coefficient found in file: " + path);
        if (n > env.shDegree || m > env.shOrder) continue;
        env.shC[(size_t)n * (n + 1) / 2 + m] = r[2];
        if (m > 0) env.shS[(size_t)n * (n + 1) / 2 + m] = r[3];
    }
    env.hasShape = true;
}

// One unit of a BRIE file: its metadata fields by name and its data.
struct BrieUnit {
    std::map<std::string, double> md;
    std::vector<double> data;
    double at(const std::string& k) const {
        auto it = md.find(k);
        if (it == md.end()) throw std::runtime_error("BRIE unit lacks metadata field '" + k + "'");
        return it->second;
    }
};

// Units of a BRIE file in either layout (brie/util/cbor.cpp:211-379).
// Layout 1: core = [{metadata: {...}, data: [...]}, ...].  Layout 2: core =
// {metadata: {nBodyUnits, intMetadata, doubleMetadata}, data: [...]}, the
// reader's member arrays written out member-major (member k of unit i at
// k * nBodyUnits + i); `intKeys` names the integer members in order ("" for
// members the reader here does not use), and the two real members are the
// start and final epochs.  Single-element array wrappers around the top-level
// map are removed, as the reference's reader does.
static std::vector<BrieUnit> brieUnits(const Value& file, const std::string& path,
                                       const std::vector<std::string>& intKeys) {
    const Value* root = &file;
    while (root->isArray() && root->size() == 1) root = &root->items()[0];
    const Value* layout = root->find("layout");
    if (!layout) throw std::runtime_error("Unknown BRIE layout type: " + path);
    std::vector<BrieUnit> out;
    if (layout->asInt() == 1) {
        for (const Value& u : root->at("core").items()) {
            BrieUnit b;
            for (const auto& kv : u.at("metadata").members())
                if (kv.second.isNumber()) b.md[kv.first] = kv.second.asDouble();
            const Value& d = u.at("data");
            b.data.resize(d.size());
            d.copyReals(0, d.size(), b.data.data());
            out.push_back(std::move(b));
        }
        return out;
    }
    if (layout->asInt() != 2)
        throw std::runtime_error("BRIE layout " + std::to_string(layout->asInt()) + " is not supported: " + path);
    const Value& core = root->at("core");
    const Value& meta = core.at("metadata");
    const int64_t n = meta.at("nBodyUnits").asInt();
    const Value& im = meta.at("intMetadata");
    const Value* dm = meta.find("doubleMetadata");
    const Value& data = core.at("data");
    const int64_t nk = (int64_t)intKeys.size();
    if (n < 0 || (int64_t)im.size() != nk * n || (dm && (int64_t)dm->size() != 2 * n))
        throw std::runtime_error("BRIE layout-2 metadata sizes do not match nBodyUnits: " + path);
    for (int64_t i = 0; i < n; ++i) {
        BrieUnit b;
        for (int64_t k = 0; k < nk; ++k)
            if (!intKeys[k].empty()) b.md[intKeys[k]] = (double)im[(size_t)(k * n + i)].asInt();
        if (dm) {
            b.md["startEpoch"] = (*dm)[(size_t)i].asDouble();
            b.md["finalEpoch"] = (*dm)[(size_t)(n + i)].asDouble();
        }
        const int64_t off = (int64_t)b.at("@offset"), size = (int64_t)b.at("@size");
        if (off < 0 || size < 0 || off + size > (int64_t)data.size())
            throw std::runtime_error("BRIE layout-2 unit data out of range: " + path);
        b.data.resize((size_t)size);
        data.copyReals((size_t)off, (size_t)size, b.data.data());
        out.push_back(std::move(b));
    }
    return out;
}

static void loadEphemeris(const std::string& path, std::vector<EphUnitHost>& out) {
    const Value root = parseCbor(readBinaryFile(path));
    // state units' integer members (brie/states/metadata/RefEphUnit.h:13-25)
    for (const BrieUnit& u : brieUnits(root, path, {"frame", "dtype", "target", "center", "nintervals", "pdeg",
                                                   "@offset", "@size"})) {
        const BrieUnit& md = u;
        if ((int)md.at("frame") != 1) throw std::runtime_error("Ephemeris units must use the ICRF frame (1): " + path);
        // Type 2: position coefficients; Type 3: position and velocity
        // coefficients (brie/core/Type3BodyUnit.h: six component blocks, the
        // position blocks first).  The force model reads positions only.
        const int64_t dtype = (int64_t)md.at("dtype");
        if (dtype != 2 && dtype != 3)
            throw std::runtime_error("Only Type-2 and Type-3 Chebyshev units are supported: " + path);
        EphUnitHost e;
        e.target = (int)md.at("target");
        e.center = (int)md.at("center");
        e.nint = (int)md.at("nintervals");
        e.pdeg = (int)md.at("pdeg");
        e.startEpoch = md.at("startEpoch");
        e.finalEpoch = md.at("finalEpoch");
        e.data = u.data;
        const size_t positions = (size_t)(1 + e.nint + 3 * (e.pdeg + 1) * e.nint);
        const size_t expected = dtype == 3 ? positions + (size_t)(3 * (e.pdeg + 1) * e.nint) : positions;
        if (e.data.size() != expected)
            throw std::runtime_error("Ephemeris unit size mismatch for target " + std::to_string(e.target));
        e.data.resize(positions);  // the velocity blocks of a Type-3 unit are not used
        out.push_back(std::move(e));
    }
}

// An Earth orientation unit of an orientation file.
struct EarthFrameUnit {
    int kind = 0, target = 0;
    int nnut = 0, nerp = 0, nint = 0, pdeg = 0, ecliptic = 0;
    int deg[3] = {0, 0, 0}, np[3] = {0, 0, 0}, barycenter = -1;  // kind 1
    int npDeg = 0, npAngles = 0;                                   // kind 2 (barycentric angles)
    double start = 0.0, final = 0.0;
    std::vector<double> data;
};

// Orientation units (brie/orientations/metadata/Layout.h:10-84,
// orientations/metadata/EphUnit.cpp:60-160): integer member 0 is the unit
// type, member 1 the rotation-data target, members 2.. depend on the type
// (IAU body models: pdeg_ra, pdeg_dec, pdeg_pm, num_dims_radii,
// barycenter, num_np_terms_ra/dec/pm; barycentric units: pdeg_np,
// num_np_angles; binary frames: inertialFrame, dtype, nintervals, pdeg;
// model units: model_id, interp_id, n_nodes_nut, n_nodes_erp,
// lag_order_nut, lag_order_erp).  Earth units are kept — the IAU model
// (target 399), the binary ITRF93 frame (3000), the IERS2000 model frame
// (3001) — with every barycentric unit; other bodies' frames are not used
// by the force model.
static void loadOrientation(const std::string& path, std::vector<EarthFrameUnit>& earth) {
    const Value root = parseCbor(readBinaryFile(path));
    const std::vector<std::string> members = {"unit_type", "@m1", "@m2", "@m3", "@m4", "@m5", "@m6", "@m7",
                                              "@m8", "@m9", "@offset", "@size"};
    for (const BrieUnit& u : brieUnits(root, path, members)) {
        // a layout-1 unit names its fields; a layout-2 unit has them by position
        auto field = [&](const char* name, const char* member) {
            auto it = u.md.find(name);
            return it != u.md.end() ? it->second : u.at(member);
        };
        const int type = (int)u.at("unit_type");
        EarthFrameUnit f;
        f.kind = type;
        f.data = u.data;
        if (type == 4) {
            f.target = (int)field("target", "@m1");
            if ((int)field("lag_order_nut", "@m6") != 5 || (int)field("lag_order_erp", "@m7") != 3)
                throw std::runtime_error("IERS2000 units must use Lagrange orders 5 (nutation) and 3 (ERP): " + path);
            f.nnut = (int)field("n_nodes_nut", "@m4");
            f.nerp = (int)field("n_nodes_erp", "@m5");
            if (f.data.size() != (size_t)(3 * f.nnut + 6 * f.nerp + 4))
                throw std::runtime_error("IERS2000 unit size mismatch: " + path);
        } else if (type == 3) {
            f.target = (int)field("frameClassID", "@m1");
            const int inertial = (int)field("inertialFrame", "@m2");
            if (inertial != 1 && inertial != 17)
                throw std::runtime_error("Binary orientation units must be relative to J2000 (1) or ECLIPJ2000 (17): "
                                         + path);
            f.ecliptic = inertial == 17;
            if ((int)field("dtype", "@m3") != 2)
                throw std::runtime_error("Binary orientation units must hold Chebyshev angles (dtype 2): " + path);
            f.nint = (int)field("nintervals", "@m4");
            f.pdeg = (int)field("pdeg", "@m5");
            if (f.nint <= 0 || f.pdeg < 0 || f.data.size() != (size_t)(1 + f.nint + 3 * (f.pdeg + 1) * f.nint))
                throw std::runtime_error("Binary orientation unit size mismatch: " + path);
        } else if (type == 1) {
            // IAU body model: RA, Dec (centuries), PM (days) polynomials in
            // degrees, nutation-precession amplitudes (RefEphUnit.h:100-330)
            f.target = (int)field("target", "@m1");
            f.deg[0] = (int)field("pdeg_ra", "@m2") + 1;
            f.deg[1] = (int)field("pdeg_dec", "@m3") + 1;
            f.deg[2] = (int)field("pdeg_pm", "@m4") + 1;
            f.barycenter = (int)field("barycenter", "@m6");
            f.np[0] = (int)field("num_np_terms_ra", "@m7");
            const auto np = [&](const char* name, int pos) {
                auto it = u.md.find(name);
                if (it != u.md.end()) return (int)it->second;
                return (int)u.at("@m" + std::to_string(pos));
            };
            f.np[1] = np("num_np_terms_dec", 8);
            f.np[2] = np("num_np_terms_pm", 9);
            size_t need = 0;
            for (int k = 0; k < 3; ++k) {
                if (f.deg[k] < 1 || f.np[k] < 0)
                    throw std::runtime_error("IAU orientation unit with invalid degrees: " + path);
                need += (size_t)(f.deg[k] + f.np[k]);
            }
            if (f.data.size() < need) throw std::runtime_error("IAU orientation unit size mismatch: " + path);
        } else if (type == 2) {
            // barycentric nutation-precession angles (degrees, centuries)
            f.target = (int)field("target", "@m1");
            f.npDeg = (int)field("pdeg_np", "@m2") + 1;
            f.npAngles = (int)field("num_np_angles", "@m3");
            if (f.npDeg < 1 || f.npAngles < 0 || f.data.size() < (size_t)(f.npDeg * f.npAngles))
                throw std::runtime_error("Barycentric orientation unit size mismatch: " + path);
            earth.push_back(std::move(f));  // kept for the body units that reference it
            continue;
        } else {
            throw std::runtime_error("Orientation unit type " + std::to_string(type) + " is not supported: " + path);
        }
        // other bodies' IAU models are kept for their J2 model
        if (f.target != 3000 && f.target != 3001 && f.target != 399 && type != 1) continue;
        if (type != 1) {
            f.start = u.at("startEpoch");
            f.final = u.at("finalEpoch");
        } else {
            f.start = -1e300;  // polynomial models hold at every epoch
            f.final = 1e300;
        }
        earth.push_back(std::move(f));
    }
}

// The Earth frame the force model uses (interface/naming/orientations
// Resolver.h:40-88, Registry.h:580-640): an explicit
// bodies.Earth.orientation picks ITRF93 (aliases ITRF, EARTH_FIXED; target
// 3000), ITRF_IERS2000 (ITRF_IPF, ITRF_NATIVE; 3001) or the IAU model
// (EARTH_BODY_FIXED, IAU_EARTH; 399); otherwise the unique loaded binary
// frame, else the IAU model.
static void selectEarthFrame(const std::vector<EarthFrameUnit>& earth, HostEnvironment& env) {
    int want = 0;
    if (!env.earthOrientation.empty()) {
        std::string n = env.earthOrientation;
        std::transform(n.begin(), n.end(), n.begin(), ::toupper);
        if (n == "ITRF93" || n == "ITRF" || n == "EARTH_FIXED") want = 3000;
        else if (n == "ITRF_IERS2000" || n == "ITRF_IPF" || n == "ITRF_NATIVE") want = 3001;
        else if (n == "EARTH_BODY_FIXED" || n == "IAU_EARTH") want = 399;
        else throw std::runtime_error("Unknown Earth orientation '" + env.earthOrientation
                                      + "'; this backend supports ITRF93, ITRF_IERS2000 and IAU_EARTH.");
    }
    const EarthFrameUnit* pick = nullptr;
    bool anyBinary = false;
    for (const EarthFrameUnit& f : earth) anyBinary |= f.target == 3000 || f.target == 3001;
    // no binary Earth frame and no explicit choice: the IAU polynomial
    if (!want && !anyBinary) want = 399;
    for (const EarthFrameUnit& f : earth) {
        if (f.kind == 2) continue;
        if (f.kind == 1 && f.target != 399) continue;  // another body's IAU model
        if (want && f.target != want) continue;
        if (!want && f.target == 399) continue;
        if (pick && pick->target != f.target)
            throw std::runtime_error("Body 399 has more than one loaded high-precision orientation frame; set "
                                     "bodies.<name>.orientation explicitly to choose between them");
        if (!pick) pick = &f;
    }
    if (want && !pick) {
        if (env.earthOrientation.empty()) return;  // no Earth orientation at all
        throw std::runtime_error("Body orientation '" + env.earthOrientation
                                 + "' needs its rotation data loaded; add the defining .brot to the "
                                   "environment's orientations");
    }
    if (!pick) return;
    env.hasRot = true;
    env.rotKind = pick->kind;
    env.rotNnut = pick->nnut;
    env.rotNerp = pick->nerp;
    env.rotNint = pick->nint;
    env.rotPdeg = pick->pdeg;
    env.rotEcliptic = pick->ecliptic;
    env.rotStart = pick->start;
    env.rotFinal = pick->final;
    env.rotData = pick->data;
    if (pick->kind == 1) {
        for (int k = 0; k < 3; ++k) {
            env.iauDeg[k] = pick->deg[k];
            env.iauNp[k] = pick->np[k];
        }
        // the body's barycentric angles, when loaded (RefEphUnit.h:670-698)
        env.iauBaryOffset = -1;
        for (const EarthFrameUnit& b : earth)
            if (b.kind == 2 && b.target == pick->barycenter) {
                int need = 0;
                for (int k = 0; k < 3; ++k) need = std::max(need, pick->np[k]);
                if (need > b.npAngles)
                    throw std::runtime_error("The barycentric orientation unit has fewer angles than the IAU model's "
                                             "nutation-precession terms.");
                env.iauBaryOffset = (int)env.rotData.size();
                env.iauNpDeg = b.npDeg;
                env.iauNpAngles = b.npAngles;
                env.rotData.insert(env.rotData.end(), b.data.begin(), b.data.end());
                break;
            }
    }
}

// The frames of the bodies other than the Earth that carry the J2 model:
// the IAU body model of the body's own NAIF id, the reference's default
// orientation target (interface/naming/orientations/Resolver.h:40-88), with
// the barycentric angles its nutation-precession terms name.
static void selectPoleFrames(const std::vector<EarthFrameUnit>& units, HostEnvironment& env) {
    env.poles.clear();
    env.shFrame = HostEnvironment::PoleBody();
    for (size_t bi = 0; bi < env.bodies.size(); ++bi) {
        const auto& b = env.bodies[bi];
        const bool field = (b.flags & kShape) != 0;
        const bool air = (b.flags & kAtmosphere) != 0;
        if (b.id == 399 || !((b.flags & kOblateness) || field || air)) continue;
        const EarthFrameUnit* pick = nullptr;
        for (const EarthFrameUnit& f : units)
            if (f.kind == 1 && f.target == b.id) {
                pick = &f;
                break;
            }
        if (!pick)
            throw std::runtime_error(std::string(field ? "The spherical-harmonic field"
                                                 : air ? "The atmosphere" : "The oblateness (J2) model")
                                     + " of " + b.name + " needs its body-fixed orientation: an IAU body model unit "
                                     "for NAIF id " + std::to_string(b.id) + " among the environment's orientations.");
        const bool pole = !field || air || (b.flags & kOblateness);
        if (pole && env.poles.size() >= (size_t)kMaxPoles)
            throw std::runtime_error("This backend takes the J2 model on at most " + std::to_string(kMaxPoles)
                                     + " bodies besides the Earth.");
        HostEnvironment::PoleBody pb;
        pb.bodyIndex = (int)bi;
        pb.data = pick->data;
        int need = 0;
        for (int k = 0; k < 3; ++k) {
            pb.deg[k] = pick->deg[k];
            pb.np[k] = pick->np[k];
            need = std::max(need, pick->np[k]);
        }
        if (need > 0)
            for (const EarthFrameUnit& u : units)
                if (u.kind == 2 && u.target == pick->barycenter) {
                    if (need > u.npAngles)
                        throw std::runtime_error("The barycentric orientation unit has fewer angles than the IAU "
                                                 "model's nutation-precession terms.");
                    pb.baryOffset = (int)pb.data.size();
                    pb.npDeg = u.npDeg;
                    pb.data.insert(pb.data.end(), u.data.begin(), u.data.end());
                    break;
                }
        if (field) env.shFrame = pb;
        if (pole) env.poles.push_back(std::move(pb));
    }
}

static double calendarMjd(int year, int month, int day) {
    const int a = (14 - month) / 12;
    const int y = year + 4800 - a;
    const int m = month + 12 * a - 3;
    const long jdn = day + (153 * m + 2) / 5 + 365L * y + y / 4 - y / 100 + y / 400 - 32045;
    return (double)jdn - 2400001.0;
}

// CelesTrak SW-All (Nrlmsise00Atmosphere.h:168-235)
static void loadSpaceWeather(const Value& nrl, HostEnvironment& env) {
    const std::string path = nrl.at("spaceWeatherFile").asString();
    const double reqStart = nrl.numberOr("coverageStartMjdUtc", -1.0);
    const double reqEnd = nrl.numberOr("coverageEndMjdUtc", -1.0);
    env.nrlHcutoff = nrl.numberOr("hCutoff", 1000.0);
    env.nrlDensityScale = nrl.numberOr("densityScale", 1.0);
    for (const auto& kv : nrl.members()) {
        std::string k = kv.first;
        std::transform(k.begin(), k.end(), k.begin(), ::tolower);
        if (k != "spaceweatherfile" && k != "coveragestartmjdutc" && k != "coverageendmjdutc" && k != "hcutoff"
            && k != "densityscale")
            throw std::runtime_error("Invalid NRLMSISE-00 atmosphere field: '" + kv.first
                                     + "'. Valid fields are: [spaceWeatherFile, coverageStartMjdUtc, "
                                       "coverageEndMjdUtc, hCutoff, densityScale].");
    }
    if (!(env.nrlHcutoff > 0.0)) throw std::runtime_error("NRLMSISE-00 hCutoff must be positive.");
    if (!(env.nrlDensityScale > 0.0)) throw std::runtime_error("NRLMSISE-00 densityScale must be positive.");
    struct Rec {
        double mjd, obs, obsc, adj, adjc, avg;
        int ap[8];
    };
    std::vector<Rec> all;
    const std::string text = readTextFile(path);
    TextLines lines(text);
    const char *lb, *le;
    while (lines.next(lb, le)) {
        LineFields ls(lb, le);
        int y, mo, d, bsrn, nd, kp[8], sumKp, c9, isn, q, avg;
        double cp, adj, adjc, adjl, obs, obsc, obsl;
        Rec r{};
        if (!(ls.readInt(y) && ls.readInt(mo) && ls.readInt(d) && ls.readInt(bsrn) && ls.readInt(nd))) continue;
        bool ok = true;
        for (int& v : kp) ok = ok && ls.readInt(v);
        ok = ok && ls.readInt(sumKp);
        for (int& v : r.ap) ok = ok && ls.readInt(v);
        ok = ok && ls.readInt(avg) && ls.readDouble(cp) && ls.readInt(c9) && ls.readInt(isn) && ls.readDouble(adj)
             && ls.readInt(q) && ls.readDouble(adjc) && ls.readDouble(adjl) && ls.readDouble(obs)
             && ls.readDouble(obsc) && ls.readDouble(obsl);
        if (!ok) continue;
        r.mjd = calendarMjd(y, mo, d);
        r.obs = obs;
        r.obsc = obsc;
        r.adj = adj;
        r.adjc = adjc;
        r.avg = avg;
        all.push_back(r);
    }
    if (all.empty()) throw std::runtime_error("No CelesTrak SW-All records found in: " + path);
    const double keepStart = reqStart >= 0.0 ? std::floor(reqStart) - 4.0 : all.front().mjd;
    const double keepEnd = reqEnd >= 0.0 ? std::floor(reqEnd) + 1.0 : all.back().mjd;
    std::vector<Rec> sel;
    for (const Rec& r : all)
        if (r.mjd >= keepStart && r.mjd <= keepEnd) sel.push_back(r);
    if (sel.size() < 5)
        throw std::runtime_error(
            "NRLMSISE-00 weather coverage is missing or too short; at least four look-back days plus the "
            "propagation day are required.");
    for (size_t i = 1; i < sel.size(); ++i)
        if (sel[i].mjd != sel[i - 1].mjd + 1.0)
            throw std::runtime_error("NRLMSISE-00 space-weather records must be consecutive days.");
    const int n = (int)sel.size();
    env.nrlNdays = n;
    env.nrlStartMjd = sel.front().mjd;
    env.nrlWeather.assign((size_t)13 * n, 0.0);
    for (int i = 0; i < n; ++i) {
        env.nrlWeather[0 * n + i] = sel[i].obs;
        env.nrlWeather[1 * n + i] = sel[i].obsc;
        env.nrlWeather[2 * n + i] = sel[i].adj;
        env.nrlWeather[3 * n + i] = sel[i].adjc;
        env.nrlWeather[4 * n + i] = sel[i].avg;
        for (int k = 0; k < 8; ++k) env.nrlWeather[(size_t)(5 + k) * n + i] = sel[i].ap[k];
    }
    env.hasNrl = true;
}

// HPOP EOP-All (earthcorrections/EarthCorrections.h:142-177)
static void loadEop(const std::string& path, HostEnvironment& env) {
    const std::string text = readTextFile(path);
    TextLines lines(text);
    const char *lb, *le;
    std::vector<std::array<double, 5>> rec;
    while (lines.next(lb, le)) {
        LineFields row(lb, le);
        int y, mo, d;
        double mjd, xp, yp, dut, lod, dpsi, deps, dx, dy, dat;
        if (!(row.readInt(y) && row.readInt(mo) && row.readInt(d) && row.readDouble(mjd) && row.readDouble(xp)
              && row.readDouble(yp) && row.readDouble(dut) && row.readDouble(lod) && row.readDouble(dpsi)
              && row.readDouble(deps) && row.readDouble(dx) && row.readDouble(dy) && row.readDouble(dat)))
            continue;
        if (!(y >= 1960 && mo >= 1 && mo <= 12 && d >= 1 && d <= 31 && std::isfinite(mjd) && std::isfinite(xp)
              && std::isfinite(yp) && std::isfinite(dut) && std::isfinite(dat) && mjd == std::floor(mjd)))
            throw std::runtime_error("Invalid Earth-tide EOP record in: " + path);
        if (!rec.empty() && mjd != rec.back()[0] + 1.0)
            throw std::runtime_error("Earth-tide EOP records must be sorted, unique, consecutive days: " + path);
        rec.push_back({mjd, xp, yp, dut, dat});
    }
    if (rec.size() < 2) throw std::runtime_error("Earth tides require at least two HPOP EOP-All records in: " + path);
    const int n = (int)rec.size();
    env.eopN = n;
    env.eopFirstMjd = rec.front()[0];
    env.eop.assign((size_t)4 * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 4; ++k) env.eop[(size_t)k * n + i] = rec[i][k + 1];
}

// Piecewise exponential atmosphere: one block or a list of blocks
// {rho0, h0, scaleHeight, hCutoff} (interface Atmosphere.h:436-508, 337-350).
static void loadExponentialAtmosphere(const Value& v, HostEnvironment& env) {
    std::vector<const Value*> blocks;
    if (v.isArray()) {
        if (v.size() == 0) throw std::runtime_error("Piecewise atmosphere list must contain at least one block.");
        for (const Value& b : v.items()) blocks.push_back(&b);
    } else if (v.isObject()) {
        blocks.push_back(&v);
    } else {
        throw std::runtime_error("Exponential atmosphere must be an object (single block) or a list of objects "
                                 "(piecewise).");
    }
    env.expSeg.clear();
    for (const Value* b : blocks) {
        if (!b->isObject()) throw std::runtime_error("Each exponential atmosphere block must be an object.");
        std::array<double, 4> seg{0.0, 0.0, 1.0, 0.0};
        bool found[4] = {false, false, false, false};
        for (const auto& kv : b->members()) {
            std::string k = kv.first;
            std::transform(k.begin(), k.end(), k.begin(), ::tolower);
            const int idx = k == "rho0" ? 0 : k == "h0" ? 1 : k == "scaleheight" ? 2 : k == "hcutoff" ? 3 : -1;
            if (idx < 0) throw std::runtime_error("Unsupported atmosphere option: " + kv.first);
            seg[idx] = kv.second.asDouble();
            found[idx] = true;
        }
        if (!found[0]) throw std::runtime_error("Atmosphere rho0 not specified.");
        if (!found[1]) throw std::runtime_error("Atmosphere h0 not specified.");
        if (!found[2]) throw std::runtime_error("Atmosphere scaleHeight not specified.");
        if (!found[3]) throw std::runtime_error("Atmosphere hCutoff not specified.");
        if (!(seg[0] >= 0.0)) throw std::runtime_error("Atmosphere rho0 must be non-negative.");
        if (!(seg[2] > 0.0)) throw std::runtime_error("Atmosphere scaleHeight must be positive.");
        env.expSeg.push_back(seg);
    }
    std::sort(env.expSeg.begin(), env.expSeg.end(), [](const auto& a, const auto& b) { return a[1] < b[1]; });
    for (size_t i = 1; i < env.expSeg.size(); ++i)
        if (!(env.expSeg[i][1] >= env.expSeg[i - 1][3]))
            throw std::runtime_error("Overlapping atmosphere segments: a band with h0=" + std::to_string(env.expSeg[i][1])
                                     + " km starts below the previous band's hCutoff="
                                     + std::to_string(env.expSeg[i - 1][3]) + " km.");
    if (env.expSeg.size() > (size_t)kMaxExpBands) throw std::runtime_error("Too many atmosphere bands for this backend.");
}

// Environment files read and parsed on threads of their own, each into a part
// of the environment that nothing else touches while it runs.  A job is
// launched at the point where a sequential load would read its file, and
// errors are reported as a sequential load meets them: a job's error, or a
// synchronous step's, gives way to the error of any job launched before it.
class FileJobs {
public:
    ~FileJobs() {
        for (Job& j : jobs_)
            if (j.thread.joinable()) j.thread.join();
    }
    size_t size() const { return jobs_.size(); }
    void launch(std::function<void()> f) {
        jobs_.emplace_back();
        Job& j = jobs_.back();
        auto run = [&j, f = std::move(f)] {
            try {
                f();
            } catch (...) {
                j.error = std::current_exception();
            }
        };
        try {
            j.thread = std::thread(run);
        } catch (const std::system_error&) {
            run();  // no thread to be had (a process limit): load this file here
        }
    }
    // Waits for jobs [0, k) and rethrows the first error among them.
    void joinUpTo(size_t k) { joinRange(0, k); }
    // Waits for jobs [a, b); on an error there, the first error of [0, b).
    void joinRange(size_t a, size_t b) {
        for (size_t i = a; i < b; ++i) join(i);
        for (size_t i = a; i < b; ++i)
            if (jobs_[i].error) {
                joinUpTo(a);
                std::rethrow_exception(jobs_[i].error);
            }
    }
    // A synchronous step failed: the first error of the jobs launched before it, else its own.
    [[noreturn]] void rethrowAfter(std::exception_ptr own) {
        joinUpTo(jobs_.size());
        std::rethrow_exception(own);
    }

private:
    struct Job {
        std::thread thread;
        std::exception_ptr error;
    };
    void join(size_t i) {
        if (jobs_[i].thread.joinable()) jobs_[i].thread.join();
    }
    std::deque<Job> jobs_;  // stable addresses: each thread writes its own Job
};

static void loadEnvironmentFiles(const Value& e, HostEnvironment& env, FileJobs& jobs);

void loadEnvironment(const Value& model, HostEnvironment& env) {
    const Value& e = model.at("environment");
    FileJobs jobs;
    try {
        loadEnvironmentFiles(e, env, jobs);
        jobs.joinUpTo(jobs.size());
    } catch (...) {
        jobs.rethrowAfter(std::current_exception());
    }
}

static void loadEnvironmentFilesIn(const Value& e, HostEnvironment& env, FileJobs& jobs,
                                   std::vector<std::vector<EphUnitHost>>& ephParts,
                                   std::vector<std::vector<EarthFrameUnit>>& oriParts);

// The per-file parts that jobs write into live here, outside the loading
// steps, and every job is joined before they go: when a synchronous step
// throws while jobs still run, the jobs never write into freed memory.
static void loadEnvironmentFiles(const Value& e, HostEnvironment& env, FileJobs& jobs) {
    std::vector<std::vector<EphUnitHost>> ephParts;
    std::vector<std::vector<EarthFrameUnit>> oriParts;
    try {
        loadEnvironmentFilesIn(e, env, jobs, ephParts, oriParts);
    } catch (...) {
        jobs.rethrowAfter(std::current_exception());
    }
}

static void loadEnvironmentFilesIn(const Value& e, HostEnvironment& env, FileJobs& jobs,
                                   std::vector<std::vector<EphUnitHost>>& ephParts,
                                   std::vector<std::vector<EarthFrameUnit>>& oriParts) {
    int shapeJobs = 0;
    for (const auto& kv : e.members()) {
        const std::string& k = kv.first;
        if (k != "bodies" && k != "ephemeris" && k != "orientations" && k != "constants" && k != "preferSSB"
            && k != "earthCorrections")
            throw std::runtime_error("Unsupported environment option: " + k);
    }
    loadConstants(e.at("constants").asString(), env);
    const Value& bodies = e.at("bodies");
    if (!bodies.isObject() || bodies.size() == 0) throw std::runtime_error("model.environment.bodies must be a nonempty object.");
    const Value* atmosphere = nullptr;
    for (const auto& kv : bodies.members()) {
        HostEnvironment::Body b;
        b.name = kv.first;
        b.id = naifId(kv.first);
        const Value& c = kv.second;
        for (const auto& f : c.members()) {
            const std::string& k = f.first;
            if (k == "gravity") {
                if (f.second.isBool()) {
                    if (f.second.asBool()) b.flags |= kGravity;
                } else if (f.second.isObject()) {
                    b.flags |= kGravity;
                    for (const auto& g : f.second.members()) {
                        std::string gk = g.first;
                        std::transform(gk.begin(), gk.end(), gk.begin(), ::tolower);
                        if (gk == "shape") {
                            if (shapeJobs && env.shBodyId != b.id)
                                throw std::runtime_error("This backend takes one spherical-harmonic field per "
                                                         "configuration; " + b.name + " would hold a second.");
                            env.shBodyId = b.id;
                            b.flags |= kShape;
                            if (shapeJobs) jobs.joinUpTo(jobs.size());  // a second table replaces the first
                            ++shapeJobs;
                            const Value* shape = &g.second;
                            jobs.launch([shape, &env] { loadShTable(*shape, env); });
                        } else if (gk == "oblateness") {
                            if (g.second.isBool() ? g.second.asBool() : !g.second.isNull()) b.flags |= kOblateness;
                        } else {
                            throw std::runtime_error("Unsupported gravity feature for " + b.name + ": " + g.first);
                        }
                    }
                } else if (f.second.isArray()) {
                    b.flags |= kGravity;
                    for (const Value& g : f.second.items()) {
                        std::string gk = g.asString();
                        std::transform(gk.begin(), gk.end(), gk.begin(), ::tolower);
                        if (gk != "oblateness")
                            throw std::runtime_error("Unsupported gravity feature for " + b.name + ": " + g.asString());
                        b.flags |= kOblateness;
                    }
                } else {
                    throw std::runtime_error("Body gravity must be a boolean or an object: " + b.name);
                }
            } else if (k == "radiation") {
                if (f.second.asBool()) {
                    if (b.id != 10) throw std::runtime_error("Radiation pressure is supported for the Sun only.");
                    b.flags |= kRadiation;
                }
            } else if (k == "occulting") {
                if (f.second.asBool()) b.flags |= kOcculting;
            } else if (k == "atmosphere") {
                // single-key model dispatch (interface Atmosphere.h:136-166);
                // NRLMSISE-00 on the Earth only (Environment.h:124-132), one
                // exponential atmosphere per configuration
                if (!f.second.isObject() || f.second.size() != 1)
                    throw std::runtime_error("Atmosphere block must be a single-key dispatch dict naming the model.");
                std::string mk = f.second.members()[0].first;
                std::transform(mk.begin(), mk.end(), mk.begin(), ::tolower);
                const Value& mv = f.second.members()[0].second;
                b.flags |= kAtmosphere;
                if (mk == "nrlmsise00" || mk == "nrlmsise-00") {
                    if (b.id != 399) throw std::runtime_error("NRLMSISE-00 may only be configured on Earth.");
                    atmosphere = &mv;
                } else if (mk == "exponential") {
                    if (!env.expSeg.empty())
                        throw std::runtime_error("This backend takes one exponential atmosphere per configuration; "
                                                 + b.name + " would hold a second.");
                    env.atmBodyId = b.id;
                    loadExponentialAtmosphere(mv, env);
                } else {
                    throw std::runtime_error("Unknown atmosphere model: '" + f.second.members()[0].first
                                             + "'.  Supported: exponential, nrlmsise00.");
                }
            } else if (k == "orientation") {
                if (b.id != 399) throw std::runtime_error("Body orientations are supported for the Earth only.");
                env.earthOrientation = f.second.asString();
            } else if (k == "flattening") {
                b.flattening = f.second.asDouble();
                if (b.id == 399) env.flattening = b.flattening;
            } else if (k == "gm") {
                b.gm = f.second.asDouble();
            } else if (k == "oblateness" || k == "shape") {
                throw std::runtime_error("Gravity sub-features (oblateness, shape) must be nested under the gravity "
                                         "block of " + b.name + ".");
            } else {
                throw std::runtime_error("Unsupported body option for " + b.name + ": " + k);
            }
        }
        if (b.gm == 0.0) {
            auto it = env.constGm.find(b.id);
            if (it != env.constGm.end()) b.gm = it->second;
            else if (b.flags & kGravity) throw std::runtime_error("No gravitational parameter for body " + b.name);
        }
        auto r = env.constRadius.find(b.id);
        b.radius = r != env.constRadius.end() ? r->second : 0.0;
        if (env.constJ2.count(b.id)) b.j2 = env.constJ2[b.id];
        if (env.constGm.count(b.id)) b.gmConst = env.constGm[b.id];
        if (env.constSoi.count(b.id)) b.soi = env.constSoi[b.id];
        env.bodies.push_back(b);
    }
    std::sort(env.bodies.begin(), env.bodies.end(), [](auto& a, auto& b) { return a.id < b.id; });
    if (env.bodies.size() > (size_t)kMaxBodies) throw std::runtime_error("Too many bodies for this backend.");
    bool haveEarth = false;
    for (auto& b : env.bodies) haveEarth |= b.id == 399;
    if (!haveEarth) throw std::runtime_error("The Earth (center of integration) must be configured.");
    // one part per file, merged in file order: a body's unit comes from the first file holding it
    if (const Value* eph = e.find("ephemeris")) {
        ephParts.resize(eph->size());
        for (size_t i = 0; i < ephParts.size(); ++i) {
            const std::string path = eph->items()[i].asString();
            std::vector<EphUnitHost>* part = &ephParts[i];
            jobs.launch([path, part] { loadEphemeris(path, *part); });
        }
    }
    {
        const size_t first = jobs.size();
        if (const Value* ori = e.find("orientations")) {
            oriParts.resize(ori->size());
            for (size_t i = 0; i < oriParts.size(); ++i) {
                const std::string path = ori->items()[i].asString();
                std::vector<EarthFrameUnit>* part = &oriParts[i];
                jobs.launch([path, part] { loadOrientation(path, *part); });
            }
        }
        jobs.joinRange(first, jobs.size());
        std::vector<EarthFrameUnit> earthFrames;
        for (auto& part : oriParts)
            for (auto& f : part) earthFrames.push_back(std::move(f));
        selectEarthFrame(earthFrames, env);
        selectPoleFrames(earthFrames, env);
    }
    if (atmosphere) jobs.launch([atmosphere, &env] { loadSpaceWeather(*atmosphere, env); });
    if (const Value* ec = e.find("earthCorrections")) {
        env.solid = ec->find("solidEarthTides") && ec->at("solidEarthTides").asBool();
        env.ocean = ec->find("oceanTides") && ec->at("oceanTides").asBool();
        env.relativity = ec->find("relativity") && ec->at("relativity").asBool();
        const std::string sys = ec->find("tideSystem") ? ec->at("tideSystem").asString() : std::string("zero_tide");
        if (sys != "zero_tide" && sys != "tide_free") throw std::runtime_error("tideSystem must be zero_tide or tide_free.");
        env.zeroTide = sys == "zero_tide";
        if (env.solid || env.ocean) {
            const std::string path = ec->at("eopFile").asString();
            jobs.launch([path, &env] { loadEop(path, env); });
        }
    }
    jobs.joinUpTo(jobs.size());
    for (auto& part : ephParts)
        for (auto& u : part) env.eph.push_back(std::move(u));
    if (((env.hasShape && env.shBodyId == 399) || env.hasNrl || env.solid || env.ocean) && !env.hasRot)
        throw std::runtime_error("An Earth orientation unit (ITRF93 or IERS2000) is required for the configured "
                                 "forces.");
}

uint64_t environmentDigest(const HostEnvironment& e) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&h](const void* p, size_t n) {
        const unsigned char* c = (const unsigned char*)p;
        for (size_t i = 0; i < n; ++i) {
            h ^= c[i];
            h *= 1099511628211ull;
        }
    };
    auto s = [&mix](const auto& x) { mix(&x, sizeof x); };
    auto v = [&mix](const auto& x) {
        const size_t n = x.size();
        mix(&n, sizeof n);
        if (n) mix(x.data(), n * sizeof(x[0]));
    };
    s(e.au);
    for (const auto* m : {&e.constGm, &e.constRadius, &e.constJ2, &e.constSoi})
        for (const auto& kv : *m) {
            s(kv.first);
            s(kv.second);
        }
    for (const auto& b : e.bodies) {
        mix(b.name.data(), b.name.size());
        s(b.id), s(b.flags), s(b.gm), s(b.radius), s(b.j2), s(b.gmConst), s(b.soi), s(b.flattening);
    }
    s(e.flattening), s(e.hasShape), s(e.shDegree), s(e.shOrder), s(e.shNormalized), s(e.shR), s(e.shGM);
    v(e.shC), v(e.shS);
    for (const auto& u : e.eph) {
        s(u.target), s(u.center), s(u.nint), s(u.pdeg), s(u.startEpoch), s(u.finalEpoch);
        v(u.data);
    }
    s(e.hasRot), s(e.rotKind), s(e.rotNnut), s(e.rotNerp), s(e.rotNint), s(e.rotPdeg), s(e.rotEcliptic);
    s(e.iauDeg), s(e.iauNp), s(e.iauBaryOffset), s(e.iauNpDeg), s(e.iauNpAngles), s(e.rotStart), s(e.rotFinal);
    v(e.rotData), v(e.expSeg);
    s(e.hasNrl), s(e.nrlStartMjd), s(e.nrlHcutoff), s(e.nrlDensityScale), s(e.nrlNdays);
    v(e.nrlWeather);
    s(e.solid), s(e.ocean), s(e.relativity), s(e.zeroTide), s(e.eopFirstMjd), s(e.eopN);
    v(e.eop);
    for (const auto& pb : e.poles) {
        s(pb.bodyIndex), s(pb.deg), s(pb.np), s(pb.baryOffset), s(pb.npDeg);
        v(pb.data);
    }
    s(e.atmBodyId), s(e.shBodyId), s(e.shFrame.bodyIndex), s(e.shFrame.deg), s(e.shFrame.np), s(e.shFrame.baryOffset);
    s(e.shFrame.npDeg), v(e.shFrame.data);
    return h;
}

// ---- engine --------------------------------------------------------------------------------------------
static int unitIndex(const HostEnvironment& env, int target) {
    for (size_t u = 0; u < env.eph.size(); ++u)
        if (env.eph[u].target == target) return (int)u;
    return -1;
}

// ephemeris units giving body - center through the common ancestor of their chains
static void chainUnits(const HostEnvironment& env, int body, int center, int plus[kMaxChain], int minus[kMaxChain]) {
    for (int k = 0; k < kMaxChain; ++k) plus[k] = minus[k] = -1;
    if (body == center) return;
    auto path = [&](int b) {
        std::vector<int> p;
        while (true) {
            p.push_back(b);
            if (b == 0) break;
            const int u = unitIndex(env, b);
            if (u < 0) throw std::runtime_error("Ephemeris does not cover body " + std::to_string(b));
            b = env.eph[u].center;
            if (p.size() > 8) throw std::runtime_error("Ephemeris chain too long");
        }
        return p;
    };
    const auto pb = path(body), pc = path(center);
    int common = 0;
    for (int x : pb)
        if (std::find(pc.begin(), pc.end(), x) != pc.end()) {
            common = x;
            break;
        }
    int np = 0, nm = 0;
    for (int x : pb) {
        if (x == common) break;
        if (np >= kMaxChain) throw std::runtime_error("Ephemeris chain too long");
        plus[np++] = unitIndex(env, x);
    }
    for (int x : pc) {
        if (x == common) break;
        if (nm >= kMaxChain) throw std::runtime_error("Ephemeris chain too long");
        minus[nm++] = unitIndex(env, x);
    }
}

template <typename T>
static T* upload(std::vector<void*>& owned, const std::vector<T>& v) {
    if (v.empty()) return nullptr;
    T* d = nullptr;
    PHOP_CUDA(cudaMalloc(&d, v.size() * sizeof(T)));
    owned.push_back(d);
    PHOP_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}

static double factorA(int n, int m, bool norm) {
    const double nn = n, mm = m;
    return norm ? std::sqrt(((2.0 * nn - 1.0) * (2.0 * nn + 1.0)) / ((nn - mm) * (nn + mm))) : (2.0 * nn - 1.0) / (nn - mm);
}
static double factorB(int n, int m, bool norm) {
    const double nn = n, mm = m;
    return norm ? std::sqrt(((2.0 * nn + 1.0) * (nn + mm - 1.0) * (nn - mm - 1.0)) / ((2.0 * nn - 3.0) * (nn + mm) * (nn - mm)))
                : (nn + mm - 1.0) / (nn - mm);
}
static double factorC(int m, bool norm) {
    if (norm) return m == 1 ? std::sqrt(3.0) : (m == 0 ? 1.0 : std::sqrt((2.0 * m + 1.0) / (2.0 * m)));
    return (m == 1 || m == 0) ? 1.0 : (2.0 * m - 1.0);
}

static std::atomic<uint64_t> g_engineSerial{0};

Engine::Engine(const HostEnvironment& env, int device) : host_(env), serial_(++g_engineSerial), device_(device) {
    PHOP_CUDA(cudaSetDevice(device_));
    PHOP_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_));
    PHOP_CUDA(cudaDeviceGetAttribute(&maxSmem_, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
    uploadEnvironment();
}

Engine::~Engine() {
    cudaSetDevice(device_);
    for (void* p : owned_) cudaFree(p);
    for (auto& kv : scratch_) cudaFree(kv.second.first);
    for (GraphEntry& g : graphs_) cudaGraphExecDestroy(g.exec);
    if (captureStream_) cudaStreamDestroy(captureStream_);
    if (gridCache_) cudaFree(gridCache_);
    if (pairCache_) cudaFree(pairCache_);
    for (auto& kv : tiles_) {
        cudaFree(kv.second.dTile);
        cudaFree(kv.second.dBlocks);
        cudaFree(kv.second.dDiagStep);
    }
}

void Engine::uploadEnvironment() {
    const HostEnvironment& h = host_;
    DevEnv& e = denv_;
    std::memset(&e, 0, sizeof e);
    e.shDegree = h.hasShape ? h.shDegree : 0;
    e.shOrder = h.hasShape ? h.shOrder : 0;
    e.shNormalized = h.shNormalized;
    e.shR = h.shR;
    e.shGM = h.shGM;
    // tide coefficients are defined with the tide model's GM and radius: they
    // join the field's low-degree block rescaled to its GM and radius, or are
    // summed on their own (scale 1) when the Earth has no gravity field file
    for (int n = 0; n <= 6; ++n)
        // in the field's units when they join the Earth's field; in the tide
        // model's own for the tides alone (no field, or a field of another body)
        e.tideScale[n] = h.hasShape && h.shBodyId == 399
                             ? (tidefield::kMuEarth * 1e-9 / h.shGM) * std::pow(tidefield::kRadius * 1e-3 / h.shR, (double)n)
                             : 1.0;
    if (h.hasShape) {
        e.shC = upload(owned_, h.shC);
        e.shS = upload(owned_, h.shS);
        LowTable low{};
        for (int n = 0; n <= kLowMax + 1 && n <= h.shDegree; ++n)
            for (int m = 0; m <= n && m <= h.shOrder; ++m) {
                const int ti = n * (n + 1) / 2 + m;
                if (n <= kLowMax) {
                    low.C[ti] = h.shC[ti];
                    low.S[ti] = h.shS[ti];
                }
                if (n > m) {
                    low.a[ti] = factorA(n, m, h.shNormalized);
                    low.b[ti] = factorB(n, m, h.shNormalized);
                }
            }
        std::vector<LowTable> lv(1, low);
        dLow_ = upload(owned_, lv);
        std::vector<double> diag((size_t)h.shOrder + 2, 0.0);
        for (int m = 0; m <= h.shOrder + 1; ++m) diag[m] = factorC(m, h.shNormalized);
        dDiag_ = upload(owned_, diag);
    }
    e.nbodies = (int)h.bodies.size();
    e.sunIndex = e.moonIndex = e.earthIndex = -1;
    int anyOcc = 0;
    for (int b = 0; b < e.nbodies; ++b) {
        const auto& B = h.bodies[b];
        e.bodyId[b] = B.id;
        e.bodyFlags[b] = B.flags;
        e.bodyGm[b] = B.gm;
        e.bodyRadius[b] = B.radius;
        e.bodyJ2[b] = B.j2;
        e.bodyGmConst[b] = B.gmConst;
        e.bodySoi[b] = B.soi;
        if (B.id == 10) e.sunIndex = b;
        if (B.id == 301) e.moonIndex = b;
        if (B.id == 399) e.earthIndex = b;
        if ((B.flags & kOcculting) && B.id != 10) anyOcc = 1;
        chainUnits(h, B.id, 399, e.chainPlus[b], e.chainMinus[b]);
    }
    e.anyOcculter = anyOcc;
    e.nExp = (int)h.expSeg.size();
    for (int k = 0; k < e.nExp; ++k)
        for (int c = 0; c < 4; ++c) e.expSeg[k][c] = h.expSeg[k][c];
    e.earthRadius = h.bodies[e.earthIndex].radius;
    e.flattening = h.flattening;
    e.atmBody = -1;
    e.atmFlattening = 0.0;
    for (size_t b = 0; b < h.bodies.size(); ++b)
        if (h.bodies[b].id == h.atmBodyId && h.atmBodyId != 399 && (h.bodies[b].flags & kAtmosphere)) {
            e.atmBody = (int)b;
            e.atmFlattening = h.bodies[b].flattening;
        }
    e.au = h.au;
    if (h.solid || h.ocean) {
        chainUnits(h, 10, 399, e.sunUnitsPlus, e.sunUnitsMinus);
        chainUnits(h, 301, 399, e.moonUnitsPlus, e.moonUnitsMinus);
    }
    e.neph = (int)h.eph.size();
    std::vector<int> nint, pdeg;
    std::vector<int64_t> off;
    std::vector<double> data;
    for (const auto& u : h.eph) {
        nint.push_back(u.nint);
        pdeg.push_back(u.pdeg);
        off.push_back((int64_t)data.size());
        data.insert(data.end(), u.data.begin(), u.data.end());
    }
    e.ephNint = upload(owned_, nint);
    e.ephPdeg = upload(owned_, pdeg);
    e.ephOffset = upload(owned_, off);
    e.ephData = upload(owned_, data);
    e.hasRot = h.hasRot;
    e.rotKind = h.rotKind;
    e.rotNnut = h.rotNnut;
    e.rotNerp = h.rotNerp;
    e.rotNint = h.rotNint;
    e.rotPdeg = h.rotPdeg;
    e.rotEcliptic = h.rotEcliptic;
    for (int k = 0; k < 3; ++k) {
        e.iauDeg[k] = h.iauDeg[k];
        e.iauNp[k] = h.iauNp[k];
    }
    e.iauBaryOffset = h.iauBaryOffset;
    e.iauNpDeg = h.iauNpDeg;
    e.iauNpAngles = h.iauNpAngles;
    e.rotData = upload(owned_, h.rotData);
    for (int b = 0; b < kMaxBodies; ++b) e.poleSlot[b] = -1;
    e.nPoles = (int)h.poles.size();
    {
        std::vector<double> coef;
        for (int k = 0; k < e.nPoles; ++k) {
            const auto& pb = h.poles[k];
            e.poleSlot[pb.bodyIndex] = k;
            for (int c = 0; c < 3; ++c) {
                e.poleDeg[k][c] = pb.deg[c];
                e.poleNp[k][c] = pb.np[c];
            }
            e.poleData[k] = (int)coef.size();
            e.poleBary[k] = pb.baryOffset;
            e.poleNpDeg[k] = pb.npDeg;
            coef.insert(coef.end(), pb.data.begin(), pb.data.end());
        }
        // a field on a body other than the Earth: its frame in every record
        e.shFrame = h.shFrame.bodyIndex >= 0 ? 1 : 0;
        if (e.shFrame) {
            for (int c = 0; c < 3; ++c) {
                e.shFrameDeg[c] = h.shFrame.deg[c];
                e.shFrameNp[c] = h.shFrame.np[c];
            }
            e.shFrameData = (int)coef.size();
            e.shFrameBary = h.shFrame.baryOffset;
            e.shFrameNpDeg = h.shFrame.npDeg;
            coef.insert(coef.end(), h.shFrame.data.begin(), h.shFrame.data.end());
        }
        e.poleCoef = coef.empty() ? nullptr : upload(owned_, coef);
    }
    // the Earth's tide deltas join the field only when it is the Earth's
    e.shTides = (h.solid || h.ocean) && h.hasShape && h.shBodyId == 399;
    e.hasNrl = h.hasNrl;
    e.nrlNdays = h.nrlNdays;
    e.nrlStartMjd = h.nrlStartMjd;
    e.nrlHcutoff = h.nrlHcutoff;
    e.nrlDensityScale = h.nrlDensityScale;
    e.nrlWeather = upload(owned_, h.nrlWeather);
    if (h.hasNrl) {
        // NRLMSISE-00 (UTC day, 3-hour slot) blocks: the weather record and ap
        // history exactly as Nrlmsise00.cu:207-235 fills them, then the
        // day/slot-only parts of the model (nrl_fast.cuh)
        const int nd = h.nrlNdays;
        std::vector<nrlf::NrlEpochBlock> blocks((size_t)nd * 8);
        const double* W = h.nrlWeather.data();
        auto at = [&](int comp, int rec) { return W[(size_t)comp * nd + rec]; };
        for (int rec = 0; rec < nd; ++rec)
            for (int slot = 0; slot < 8; ++slot) {
                nrlf::NrlEpochBlock& b = blocks[(size_t)rec * 8 + slot];
                std::memset(&b, 0, sizeof b);
                if (rec < 3) continue;
                auto lag = [&](int l) {
                    const int hh = 24 + slot - l;
                    return at(5 + hh % 8, rec - 3 + hh / 8);
                };
                double apa[7];
                apa[0] = at(4, rec);
                apa[1] = at(5 + slot, rec);
                apa[2] = lag(1);
                apa[3] = lag(2);
                apa[4] = lag(3);
                apa[5] = apa[6] = 0.0;
                for (int d = 4; d <= 11; ++d) apa[5] += lag(d);
                for (int d = 12; d <= 19; ++d) apa[6] += lag(d);
                apa[5] /= 8.0;
                apa[6] /= 8.0;
                // day of year of the record's UTC date (calendarDate, Nrlmsise00.cu:113-130)
                const double mjd = h.nrlStartMjd + rec;
                const long a = (long)std::floor(mjd + 2400001.0);
                long bb = 0, c = 0;
                if (a < 2299161) c = a + 1524;
                else {
                    bb = (long)((a - 1867216.25) / 36524.25);
                    c = a + bb - bb / 4 + 1525;
                }
                const long dd = (long)((c - 122.1) / 365.25);
                const long ee = 365 * dd + dd / 4;
                const long ff = (long)((c - ee) / 30.6001);
                const int day = (int)(c - ee - (long)(30.6001 * ff));
                const int month = (int)(ff - 1 - 12 * (ff / 14));
                const int year = (int)(dd - 4715 - (7 + month) / 10);
                int mdays[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
                if ((year % 4 == 0 && year % 100 != 0) || year % 400 == 0) mdays[1] = 29;
                int doy = day;
                for (int m = 1; m < month; ++m) doy += mdays[m - 1];
                nrlf::nrlSlotBlock(doy, at(2, rec - 1), at(3, rec), apa, b);
                if (!b.valid)
                    throw std::runtime_error("NRLMSISE-00: a coefficient table outside pt / pd[0] has a "
                                             "latitude-dependent ap response; this backend does not support it.");
            }
        e.nrlBlocks = upload(owned_, blocks);
    }
    e.solid = h.solid;
    e.ocean = h.ocean;
    e.relativity = h.relativity;
    e.tidesAlone = (h.solid || h.ocean) && !(h.hasShape && h.shBodyId == 399);
    e.zeroTide = h.zeroTide;
    e.tideOcean = nullptr;
    if (h.ocean) {
        std::vector<tidefield::OceanAmp> ocean(tidefield::kWaves * tidefield::kSlots);
        tidefield::buildOceanTable(ocean.data());
        e.tideOcean = upload(owned_, ocean);
    }
    e.eopN = h.eopN;
    e.eopFirstMjd = h.eopFirstMjd;
    e.eop = upload(owned_, h.eop);
}

// Lane-interleaved coefficient tile for the n > 8 part (layout in propagate.cuh)
const Engine::Tile& Engine::tileFor(int L, bool split, int lowDeg) {
    const int key = (lowDeg * 32 + L) * 2 + (split ? 1 : 0);
    auto it = tiles_.find(key);
    if (it != tiles_.end()) return it->second;
    const HostEnvironment& h = host_;
    const int N = h.shDegree, M = h.shOrder;
    const bool norm = h.shNormalized != 0;
    const int nb = h.hasShape ? (M + 1 + L - 1) / L : 0;
    std::vector<int2> blocks(nb > 0 ? nb : 1, int2{0, 0});
    std::vector<TileD> entries;
    for (int b = 0; b < nb; ++b) {
        const int n0b = std::max(b * L, lowDeg + 1);
        const int len = std::max(0, N - n0b + 1);
        blocks[b] = int2{(int)entries.size(), len};
        const size_t base = entries.size();
        entries.resize(base + (size_t)len * L, TileD{0, 0, 0, 0, 0, 0});
        for (int j = 0; j < L; ++j) {
            const int m = b * L + j;
            if (m > M) continue;
            const int n0 = std::max(m, lowDeg + 1);
            for (int i = 0; i < len; ++i) {
                const int n = n0 + i;
                if (n > N) break;
                TileD& t = entries[base + (size_t)i * L + j];
                const size_t ti = (size_t)n * (n + 1) / 2 + m;
                t.c = h.shC[ti];
                t.s = m > 0 ? h.shS[ti] : 0.0;
                t.cp = (double)(n + 1) * t.c;
                t.sp = (double)(n + 1) * t.s;
                if (n + 1 <= N) {
                    t.a = factorA(n + 1, m, norm);
                    t.b = factorB(n + 1, m, norm);
                }
            }
        }
    }
    Tile tile;
    tile.nblocks = nb;
    std::vector<unsigned char> bytes;
    if (split) {
        std::vector<TileF> f(entries.size());
        for (size_t k = 0; k < entries.size(); ++k)
            f[k] = TileF{(float)entries[k].c, (float)entries[k].s, (float)entries[k].cp, (float)entries[k].sp,
                         (float)entries[k].a, (float)entries[k].b, 0.f, 0.f};
        bytes.resize(f.size() * sizeof(TileF));
        std::memcpy(bytes.data(), f.data(), bytes.size());
    } else {
        bytes.resize(entries.size() * sizeof(TileD));
        std::memcpy(bytes.data(), entries.data(), bytes.size());
    }
    bytes.resize((bytes.size() + 15) / 16 * 16 + 16, 0);
    tile.bytes = (int)bytes.size();
    PHOP_CUDA(cudaMalloc(&tile.dTile, bytes.size()));
    PHOP_CUDA(cudaMemcpy(tile.dTile, bytes.data(), bytes.size(), cudaMemcpyHostToDevice));
    PHOP_CUDA(cudaMalloc(&tile.dBlocks, blocks.size() * sizeof(int2)));
    PHOP_CUDA(cudaMemcpy(tile.dBlocks, blocks.data(), blocks.size() * sizeof(int2), cudaMemcpyHostToDevice));
    // diagonal block factors D_m = c_{m+1} ... c_{m+L} and D_m (m+L)/m
    std::vector<double2> diagStep((size_t)M + 1, double2{0.0, 0.0});
    for (int m = 0; m + L <= M; ++m) {
        double d = 1.0;
        for (int k = m + 1; k <= m + L; ++k) d *= factorC(k, norm);
        diagStep[m] = double2{d, m > 0 ? d * ((double)(m + L) / (double)m) : d};
    }
    PHOP_CUDA(cudaMalloc(&tile.dDiagStep, diagStep.size() * sizeof(double2)));
    PHOP_CUDA(cudaMemcpy(tile.dDiagStep, diagStep.data(), diagStep.size() * sizeof(double2), cudaMemcpyHostToDevice));
    return tiles_.emplace(key, tile).first->second;
}

void* Engine::scratch(const std::string& name, size_t bytes) {
    auto it = scratch_.find(name);
    if (it != scratch_.end() && it->second.second >= bytes) return it->second.first;
    if (it != scratch_.end()) {
        cudaFree(it->second.first);
        scratch_.erase(it);
    }
    void* p = nullptr;
    PHOP_CUDA(cudaMalloc(&p, bytes > 0 ? bytes : 16));
    scratch_[name] = {p, bytes};
    return p;
}

int Engine::autoLanes(int64_t n) const {
    // enough threads for ~16 resident warps per SM, at most 16 lanes per object
    const double want = (double)sms_ * 512.0 / (double)std::max<int64_t>(n, 1);
    int L = 1;
    while (L < 16 && L < want) L *= 2;
    return L;
}

void Engine::assertCoverage(double loMjd, double hiMjd) const {
    const double lo = mjdToEtHost(loMjd), hi = mjdToEtHost(hiMjd);
    for (const auto& u : host_.eph)
        if (lo < u.startEpoch || hi > u.finalEpoch)
            throw std::runtime_error("Ephemeris coverage is insufficient for the requested epochs (target "
                                     + std::to_string(u.target) + ").");
    if (host_.hasRot && (lo < host_.rotStart || hi > host_.rotFinal))
        throw std::runtime_error("Earth orientation coverage is insufficient for the requested epochs.");
}

// ---- scheduling ---------------------------------------------------------------------------------
// Objects whose altitudes are close take the same branches through the
// NRLMSISE-00 model (lower / upper thermosphere, cut-off), so the work queue
// hands them out in order of geocentric radius: warps stay converged and the
// results do not depend on the order (objects never interact).
__global__ void radiusKeysKernel(const double* __restrict__ state, int64_t stride, const int64_t* __restrict__ slots,
                                 int64_t n, uint32_t* __restrict__ keys, int64_t* __restrict__ idx) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t o = slots ? slots[i] : i;
    const double x = state[o], y = state[stride + o], z = state[2 * stride + o];
    const float r2 = (float)(x * x + y * y + z * z);
    keys[i] = isfinite(r2) ? __float_as_uint(r2) : 0xffffffffu;  // non-negative floats order as integers
    idx[i] = o;
}

const int64_t* Engine::orderByRadius(int64_t n, const double* dState, cudaStream_t stream, int64_t* launches,
                                     int64_t stride, const int64_t* slots) {
    if (n > INT32_MAX) throw std::runtime_error("too many objects for one batch");
    uint32_t* keys = (uint32_t*)scratch("orderKeys", (size_t)n * 4);
    uint32_t* keysOut = (uint32_t*)scratch("orderKeysOut", (size_t)n * 4);
    int64_t* idx = (int64_t*)scratch("orderIdx", (size_t)n * 8);
    int64_t* order = (int64_t*)scratch("order", (size_t)n * 8);
    radiusKeysKernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(dState, stride ? stride : n, slots, n, keys, idx);
    PHOP_CUDA(cudaGetLastError());
    size_t temp = 0;
    PHOP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, keys, keysOut, idx, order, (int)n, 0, 32, stream));
    void* dTemp = scratch("orderTemp", temp);
    PHOP_CUDA(cub::DeviceRadixSort::SortPairs(dTemp, temp, keys, keysOut, idx, order, (int)n, 0, 32, stream));
    if (launches) *launches += 1 + 6;  // key kernel + CUB histogram, scan and four one-sweep passes (32-bit keys)
    return order;
}

// Epoch records at TDB seconds k * 30 for every k whose 4-point stencil an
// epoch in [lo, hi] can reach, for the per-object time path.  Records depend
// on the absolute epoch alone, so the context keeps them: a request inside
// the kept range reuses it, one beyond it extends the range (with a margin of
// a quarter of the span, at least a day, so that slices that advance a batch
// step by step rarely extend it again) and computes only the new records.
void Engine::buildRecordGrid(double lo, double hi, TimeGrid& g, cudaStream_t stream, int64_t* launches) {
    const double H = kRecordGridSeconds;
    const int64_t kLo = (int64_t)std::floor(lo / H) - 1;
    const int64_t kHi = (int64_t)std::ceil(hi / H) + 2;
    if (kHi - kLo + 1 > (int64_t)1 << 26) throw std::runtime_error("the batch spans too long a time interval");
    if (!(gridCache_ && kLo >= gridKLo_ && kHi <= gridKHi_)) {
        const int64_t margin = std::max<int64_t>(2880, (kHi - kLo) / 4);
        int64_t a = kLo, b = kHi + margin;
        if (gridCache_ && gridKHi_ >= a - 1 && gridKLo_ <= b + 1) {  // overlapping or adjacent: keep the old records
            a = std::min(a, gridKLo_);
            b = std::max(b, gridKHi_);
        }
        const int64_t G = b - a + 1;
        if (G > (int64_t)1 << 26) throw std::runtime_error("the batch spans too long a time interval");
        EpochRecord* fresh = nullptr;
        PHOP_CUDA(cudaMalloc(&fresh, (size_t)G * sizeof(EpochRecord)));
        std::vector<double> ts;
        std::vector<int64_t> at;  // grid indices to compute
        const bool keep = gridCache_ && gridKLo_ >= a && gridKHi_ <= b;
        for (int64_t k = a; k <= b; ++k)
            if (!(keep && k >= gridKLo_ && k <= gridKHi_)) at.push_back(k);
        if (keep) {
            PHOP_CUDA(cudaMemcpyAsync(fresh + (gridKLo_ - a), gridCache_,
                                      (size_t)(gridKHi_ - gridKLo_ + 1) * sizeof(EpochRecord),
                                      cudaMemcpyDeviceToDevice, stream));
        }
        // the new records come in at most two contiguous runs (below and above the kept range)
        size_t i = 0;
        while (i < at.size()) {
            size_t j = i;
            while (j + 1 < at.size() && at[j + 1] == at[j] + 1) ++j;
            const int64_t count = (int64_t)(j - i + 1);
            ts.resize(count);
            for (int64_t q = 0; q < count; ++q) ts[q] = (double)(at[i] + q) * H;
            double* dT = (double*)scratch("gridT", (size_t)count * 8);
            PHOP_CUDA(cudaMemcpyAsync(dT, ts.data(), (size_t)count * 8, cudaMemcpyHostToDevice, stream));
            launchEpochRecords(denv_, dT, (int)count, fresh + (at[i] - a), stream);
            PHOP_CUDA(cudaGetLastError());
            PHOP_CUDA(cudaStreamSynchronize(stream));  // ts is reused by the next run
            if (launches) *launches += 1;
            i = j + 1;
        }
        if (gridCache_) {
            PHOP_CUDA(cudaStreamSynchronize(stream));
            cudaFree(gridCache_);
        }
        gridCache_ = fresh;
        gridKLo_ = a;
        gridKHi_ = b;
        if (pairCache_) cudaFree(pairCache_);
        pairCache_ = nullptr;
        PHOP_CUDA(cudaMalloc(&pairCache_, (size_t)(G - 1) * kInterpFields * sizeof(double2)));
        launchRecordPairs(gridCache_, G, pairCache_, stream);
        PHOP_CUDA(cudaGetLastError());
        if (launches) *launches += 1;
    }
    g.grid = gridCache_;
    g.gridPairs = pairCache_;
    g.gridH = H;
    g.gridBase = gridKLo_;
    g.gridN = (int)(gridKHi_ - gridKLo_ + 1);
}

Engine::LaunchShape Engine::launchStep(StepParams p, int L, const RunOptions& opt, bool shared, cudaStream_t stream) {
    const LaunchShape shape = prepareStep(p, L, opt, shared);
    enqueueStep(p, shape, opt, shared, stream);
    return shape;
}

void Engine::enqueueStep(const StepParams& p, const LaunchShape& shape, const RunOptions& opt, bool shared,
                         cudaStream_t stream) {
    PHOP_CUDA(cudaMemsetAsync(p.workCounter, 0, 2 * sizeof(int), stream));
    PHOP_CUDA(launchPropagate(p, shape.lanes, opt.split, shared, shape.ctas, shape.threads, stream));
}

// The step launch (control-word reset + step kernel) as a CUDA graph, cached
// by its exact launch parameters: repeated batches of the same shape replay
// the instantiated graph instead of issuing the launch sequence again.
void Engine::launchStepGraph(const StepParams& p, const LaunchShape& shape, const RunOptions& opt, bool shared,
                             cudaStream_t stream) {
    GraphEntry key;
    std::memcpy(key.params, &p, sizeof(StepParams));
    key.lanes = shape.lanes;
    key.threads = shape.threads;
    key.ctas = shape.ctas;
    key.flags = (opt.split ? 1 : 0) | (shared ? 2 : 0);
    for (const GraphEntry& g : graphs_)
        if (g.lanes == key.lanes && g.threads == key.threads && g.ctas == key.ctas && g.flags == key.flags
            && std::memcmp(g.params, key.params, sizeof(StepParams)) == 0) {
            PHOP_CUDA(cudaGraphLaunch(g.exec, stream));
            return;
        }
    if (graphs_.size() >= 16) {
        for (GraphEntry& g : graphs_) cudaGraphExecDestroy(g.exec);
        graphs_.clear();
    }
    // captured on the engine's own stream (the legacy default stream cannot
    // be captured); the instantiated graph is launched on the caller's stream
    if (!captureStream_) PHOP_CUDA(cudaStreamCreateWithFlags(&captureStream_, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    PHOP_CUDA(cudaStreamBeginCapture(captureStream_, cudaStreamCaptureModeRelaxed));
    try {
        enqueueStep(p, shape, opt, shared, captureStream_);
    } catch (...) {
        cudaStreamEndCapture(captureStream_, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    PHOP_CUDA(cudaStreamEndCapture(captureStream_, &graph));
    const cudaError_t ie = cudaGraphInstantiate(&key.exec, graph, 0);
    cudaGraphDestroy(graph);
    PHOP_CUDA(ie);
    graphs_.push_back(key);
    PHOP_CUDA(cudaGraphLaunch(key.exec, stream));
}

// FP64 low part of each column: n <= 8 in the FP64 form, n <= the option's
// degree in split precision.  Its default follows the field's degree: the
// FP32 rounding of the recursion accumulates over more terms in a larger
// field (24 h, 10^5 LEO objects at degree 120: 11.5 mm max with n <= 20 in
// FP64, 8.3 mm with n <= 24; degree 70: 6.4 mm with n <= 20).
int lowDegreeFor(const RunOptions& opt, int fieldDegree) {
    if (!opt.split) return kLowDeg;
    const int d = opt.splitFp64Degree > 0 ? opt.splitFp64Degree
                                          : (fieldDegree > 80 ? kSplitFp64DegreeHigh : kSplitFp64Degree);
    return d < kLowDeg ? kLowDeg : (d > kLowMax ? kLowMax : d);
}

// Host side of a launch: coefficient tile, shared-memory split and grid.
Engine::LaunchShape Engine::prepareStep(StepParams& p, int L, const RunOptions& opt, bool shared) {
    if (L != 1 && L != 2 && L != 4 && L != 8 && L != 16) throw std::runtime_error("lanes must be 1, 2, 4, 8 or 16");
    const int lowDeg = lowDegreeFor(opt, host_.shDegree);
    // lane-group pairs share the tile (built for 2L lanes); not with the
    // split form's FP64 floor, whose low objects take the FP64 tile of L lanes
    const bool pair = opt.pairSh < 0 ? L <= 4 : opt.pairSh != 0;
    p.pairSh = (pair && L <= 4 && !(opt.split && opt.splitFloorKm > 0.0)) ? 1 : 0;
    p.deepRegs = (opt.deepRegs > 0 && hasDeepShape(L)) ? 1 : 0;
    const Tile& tile = tileFor(p.pairSh ? 2 * L : L, opt.split, lowDeg);
    p.tile = tile.dTile;
    p.tileBytes = tile.bytes;
    p.blocks = tile.dBlocks;
    p.nblocks = tile.nblocks;
    p.diagStep = tile.dDiagStep;
    p.lowDeg = lowDeg;
    p.tile64 = nullptr;
    p.splitRadius = 0.0;
    if (opt.split && opt.splitFloorKm > 0.0) {
        p.tile64 = tileFor(L, false, lowDeg).dTile;
        p.splitRadius = host_.shR + opt.splitFloorKm;
    }
    // shared memory per CTA: the coefficient tile (when it fits) plus the
    // stage derivatives, 13 x ceil(6/L) doubles per thread
    int registers = 0;
    int threadsReq = std::min(opt.threads > 0 ? opt.threads : 512, stepThreadBound(L, p.deepRegs));
    {
        // never more threads than the compiled instantiation accepts (its
        // register count times the threads must fit the SM's register file)
        const int akey = (((L * 2 + (opt.split ? 1 : 0)) * 2 + (shared ? 1 : 0)) * 2 + p.pairSh) * 2 + p.deepRegs;
        auto at = attrs_.find(akey);
        if (at == attrs_.end()) {
            cudaFuncAttributes a{};
            PHOP_CUDA(propagateAttributes(L, opt.split, shared, p.pairSh, p.deepRegs, &a));
            at = attrs_.emplace(akey, std::make_pair(a.maxThreadsPerBlock, a.numRegs)).first;
        }
        threadsReq = std::max(32, std::min(threadsReq, at->second.first / 32 * 32));
        registers = at->second.second;
    }
    const int kPerThread = 13 * ((6 + L - 1) / L) * 8;
    int threads = threadsReq;
    if (opt.tileSmem != 0 && tile.bytes + 1024 + 64 * kPerThread <= maxSmem_) {
        p.useSmemTile = 1;
        threads = std::min(threadsReq, (maxSmem_ - tile.bytes - 1024) / kPerThread / 32 * 32);
    } else {
        p.useSmemTile = 0;
        threads = std::min(threadsReq, (maxSmem_ - 1024) / kPerThread / 32 * 32);
    }
    int perSm = opt.ctasPerSm;
    if (perSm <= 0) {
        const int smem = propagateSmemBytes(p, L, threads);
        const int64_t key = (((((int64_t)smem * 1024 + threads) * 32 + L) * 4 + (opt.split ? 2 : 0) + (shared ? 1 : 0)) * 2
                             + p.pairSh) * 2 + p.deepRegs;
        auto it = occupancy_.find(key);
        if (it == occupancy_.end())
            it = occupancy_
                     .emplace(key, propagateMaxCtasPerSm(L, opt.split, shared, p.pairSh, p.deepRegs, threads, smem))
                     .first;
        perSm = it->second;
    }
    if (perSm <= 0) perSm = 1;
    // one warp per group of 32 / L objects; when every group fits one wave,
    // spread the warps evenly over all SMs instead of filling CTAs first
    const int64_t warpsNeeded = (p.n + (32 / L) - 1) / (32 / L);
    const int64_t slots = (int64_t)sms_ * perSm;
    if (warpsNeeded <= slots * (threads / 32)) {
        const int64_t warpsPerCta = (warpsNeeded + slots - 1) / slots;
        threads = (int)std::min<int64_t>(threads, std::max<int64_t>(1, warpsPerCta) * 32);
    }
    const int64_t warpsPerCta = threads / 32;
    const int64_t need = (warpsNeeded + warpsPerCta - 1) / warpsPerCta;
    LaunchShape shape;
    shape.lanes = L;
    shape.threads = threads;
    shape.ctas = (int)std::max<int64_t>(1, std::min<int64_t>(slots, need));
    shape.smemTile = p.useSmemTile != 0;
    shape.registers = registers;
    return shape;
}

// Project autotuner for the launch shape: lanes per object (1, 2, 4, 8, 16),
// objects per lane in the geopotential (one, or two for lane-group pairs at
// up to four lanes) and, at two and four lanes, the thread bound the kernel
// is compiled for (wide: 320 / 384 threads at 168 registers; deep: 256
// threads at 255 registers).  Threads per CTA follow from the bound, shared
// memory and the batch size (prepareStep).  The first batch of each class
// (log2 of the batch size, time-grid mode, precision, pairing and bound
// options) times a short probe of
// every shape on scratch copies of the inputs and keeps the fastest; later
// batches of the class reuse the choice.  A probe launch advances every
// object by up to twelve steps, fewer for large batches so that one launch
// stays near kProbeObjectSteps object-steps (at least one step); the
// fastest of two timed launches after an untimed warm-up counts.
// PARAHPOP_B200_TUNE_LOG=1 prints the probe times.
static constexpr int64_t kProbeObjectSteps = int64_t(1) << 17;
int Engine::tunedShape(const StepParams& base, const RunOptions& opt, bool shared, cudaStream_t stream,
                       int64_t* launches) {
    int bucket = 0;
    while (bucket < 40 && (int64_t(1) << bucket) < base.n) ++bucket;
    const int key = ((bucket * 4 + (shared ? 2 : 0) + (opt.split ? 1 : 0)) * 4 + (opt.pairSh + 1)) * 4
                    + (opt.deepRegs + 1);
    auto it = tuned_.find(key);
    if (it != tuned_.end()) return it->second;
    if (base.stride != 0 && base.stride != base.n) {  // pools pin their lane count
        const int L = autoLanes(base.n);
        const int pair = opt.pairSh < 0 ? (L <= 4 ? 1 : 0) : opt.pairSh;
        return (L * 2 + pair) * 2 + (opt.deepRegs > 0 && hasDeepShape(L) ? 1 : 0);
    }
    const int64_t n = base.n;
    StepParams p = base;
    double* st = (double*)scratch("probeState", (size_t)6 * n * 8);
    p.state = st;
    const int probeSteps = (int)std::max<int64_t>(1, std::min<int64_t>(12, kProbeObjectSteps / std::max<int64_t>(1, n)));
    if (shared) {
        p.nsteps = std::min(p.nsteps, probeSteps);
    } else {
        p.maxSteps = probeSteps;
        p.cur = (double*)scratch("probeCur", (size_t)n * 8);
        p.dt = (double*)scratch("probeDt", (size_t)n * 8);
        p.unfinished = (int*)scratch("probeUnf", (size_t)n * 4);
    }
    cudaEvent_t e0, e1;
    PHOP_CUDA(cudaEventCreate(&e0));
    PHOP_CUDA(cudaEventCreate(&e1));
    int best = (autoLanes(n) * 2 + (opt.pairSh > 0 ? 1 : 0)) * 2;
    float bestMs = 1e30f;
    const char* logEnv = std::getenv("PARAHPOP_B200_TUNE_LOG");
    const bool tuneLog = logEnv && std::atoi(logEnv) != 0;
    // shape code: ((lanes * 2 + pairs) * 2 + deep thread bound)
    for (int code = 4; code < 68; ++code) {
        const int L = code >> 2, pair = (code >> 1) & 1, deep = code & 1;
        if (L != 1 && L != 2 && L != 4 && L != 8 && L != 16) continue;
        if (opt.pairSh >= 0 && pair != opt.pairSh) continue;
        if (opt.pairSh < 0 && pair && L >= 8) continue;  // pairs at 8 and 16 lanes measured slower on every workload
        if (deep && !hasDeepShape(L)) continue;
        if (opt.deepRegs >= 0 && deep != (opt.deepRegs && hasDeepShape(L) ? 1 : 0)) continue;
        if (L >= 8 && n >= (int64_t)sms_ * 512 * 4) continue;  // enough objects to fill the GPU with narrow groups
        RunOptions o = opt;
        o.pairSh = pair;
        o.deepRegs = deep;
        // an untimed launch first (module loading, attribute set-up), then the
        // fastest of two timed probes
        float ms = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            PHOP_CUDA(cudaMemcpyAsync(st, base.state, (size_t)6 * n * 8, cudaMemcpyDeviceToDevice, stream));
            if (!shared) {
                PHOP_CUDA(cudaMemcpyAsync(p.cur, base.cur, (size_t)n * 8, cudaMemcpyDeviceToDevice, stream));
                PHOP_CUDA(cudaMemcpyAsync(p.dt, base.dt, (size_t)n * 8, cudaMemcpyDeviceToDevice, stream));
            }
            StepParams q = p;
            const LaunchShape shape = prepareStep(q, L, o, shared);
            PHOP_CUDA(cudaEventRecord(e0, stream));
            enqueueStep(q, shape, o, shared, stream);
            PHOP_CUDA(cudaEventRecord(e1, stream));
            PHOP_CUDA(cudaEventSynchronize(e1));
            if (launches) ++*launches;
            float t = 0.f;
            PHOP_CUDA(cudaEventElapsedTime(&t, e0, e1));
            if (rep > 0) ms = std::min(ms, t);
        }
        int err = 0;
        PHOP_CUDA(cudaMemcpy(&err, p.errorFlag, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) throw std::runtime_error("Propagation kernel reported error " + std::to_string(err) + ".");
        if (tuneLog)
            std::fprintf(stderr,
                         "parahpop-b200 tune: n=%lld shared=%d split=%d lanes=%d pairs=%d deep=%d probe_steps=%d "
                         "probe_ms=%.3f\n",
                         (long long)n, shared ? 1 : 0, opt.split ? 1 : 0, L, pair, deep, probeSteps, ms);
        if (ms < bestMs) {
            bestMs = ms;
            best = code;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tuned_[key] = best;
    return best;
}

void Engine::runKernel(int64_t n, double* dState, const double* dBc, const double* dAms, const TimeGrid& g,
                       const int64_t* dOrder, int64_t maxSteps, const RunOptions& opt, RunStats* stats,
                       cudaStream_t stream, int64_t launchesBefore) {
    StepParams p{};
    p.env = denv_;
    p.n = n;
    p.state = dState;
    p.bc = dBc;
    p.ams = dAms;
    p.low = dLow_;
    p.diagC = dDiag_;
    p.maxSteps = maxSteps;
    p.order = dOrder;
    p.cur = g.cur;
    p.end = g.end;
    p.dt = g.dt1;
    p.step = g.step;
    p.unfinished = g.unfinished;
    p.grid = g.grid;
    p.gridPairs = g.gridPairs;
    p.gridH = g.gridH;
    p.gridBase = g.gridBase;
    p.gridN = g.gridN;
    p.stride = g.stride;
    const bool shared = g.shared;
    cudaEvent_t e0, e1, e2, eTuned;
    PHOP_CUDA(cudaEventCreate(&e0));
    PHOP_CUDA(cudaEventCreate(&e1));
    PHOP_CUDA(cudaEventCreate(&e2));
    PHOP_CUDA(cudaEventCreate(&eTuned));
    int64_t launches = launchesBefore;
    PHOP_CUDA(cudaEventRecord(e0, stream));
    if (shared) {
        const int nsteps = (int)g.t0.size();
        std::vector<double> stageT((size_t)nsteps * 13);
        static const double c[12] = {2. / 27, 1. / 9, 1. / 6, 5. / 12, 1. / 2, 5. / 6, 1. / 6, 2. / 3, 1. / 3, 1.0, 0, 1.0};
        for (int k = 0; k < nsteps; ++k)
            for (int s = 0; s < 13; ++s)
                stageT[(size_t)k * 13 + s] = s == 0 ? g.t0[k] : std::fma(g.dt[k], c[s - 1], g.t0[k]);
        double* dStage = (double*)scratch("stageT", stageT.size() * sizeof(double));
        EpochRecord* dRec = (EpochRecord*)scratch("records", stageT.size() * sizeof(EpochRecord));
        double* dT0 = (double*)scratch("t0", (size_t)nsteps * sizeof(double));
        double* dDtv = (double*)scratch("dt", (size_t)nsteps * sizeof(double));
        PHOP_CUDA(cudaMemcpyAsync(dStage, stageT.data(), stageT.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        PHOP_CUDA(cudaMemcpyAsync(dT0, g.t0.data(), (size_t)nsteps * sizeof(double), cudaMemcpyHostToDevice, stream));
        PHOP_CUDA(cudaMemcpyAsync(dDtv, g.dt.data(), (size_t)nsteps * sizeof(double), cudaMemcpyHostToDevice, stream));
        launchEpochRecords(denv_, dStage, (int)stageT.size(), dRec, stream);
        PHOP_CUDA(cudaGetLastError());
        ++launches;
        p.nsteps = nsteps;
        p.stepT0 = dT0;
        p.stepDt = dDtv;
        p.records = dRec;
    }
    if (opt.dTraj && (!shared || opt.trajEvery <= 0))
        throw std::runtime_error("Trajectory records need a batch with one epoch, duration and step.");
    int* dCtl = (int*)scratch("ctl", 4 * sizeof(int));
    p.workCounter = dCtl;
    p.errorFlag = dCtl + 1;
    p.tileFallbacks = dCtl + 2;
    p.tileWaitTest = opt.tileWaitTest;
    PHOP_CUDA(cudaMemsetAsync(dCtl, 0, 4 * sizeof(int), stream));
    PHOP_CUDA(cudaEventRecord(eTuned, stream));  // end of the epoch records
    RunOptions o = opt;
    int L = opt.lanes;
    if (L <= 0) {
        const int code = tunedShape(p, opt, shared, stream, &launches);
        L = code >> 2;
        o.pairSh = (code >> 1) & 1;
        o.deepRegs = code & 1;
    }
    if (opt.dTraj) {  // after the autotuner's probes, which must not write records
        p.traj = opt.dTraj;
        p.trajEvery = opt.trajEvery;
        p.trajRecords = opt.trajRecords;
    }
    const LaunchShape shape = prepareStep(p, L, o, shared);
    PHOP_CUDA(cudaEventRecord(e1, stream));
    if (opt.graph) launchStepGraph(p, shape, o, shared, stream);
    else enqueueStep(p, shape, o, shared, stream);
    ++launches;
    PHOP_CUDA(cudaEventRecord(e2, stream));
    PHOP_CUDA(cudaEventSynchronize(e2));
    int ctl[3] = {0, 0, 0};
    PHOP_CUDA(cudaMemcpy(ctl, dCtl, 3 * sizeof(int), cudaMemcpyDeviceToHost));
    const int err = ctl[1];
    if (err) throw std::runtime_error("Propagation kernel reported error " + std::to_string(err) + ".");
    if (stats) {
        stats->tileFallbacks += ctl[2];
        float a = 0, b = 0, c = 0;
        cudaEventElapsedTime(&a, e0, eTuned);
        cudaEventElapsedTime(&c, eTuned, e1);
        cudaEventElapsedTime(&b, e1, e2);
        stats->recordsMs += a;
        stats->tuneMs += c;
        stats->kernelMs += b;
        stats->launches += launches;
        stats->lanes = shape.lanes;
        stats->ctas = shape.ctas;
        stats->threads = shape.threads;
        stats->split = opt.split;
        stats->sharedGrid = shared;
        stats->tileInSmem = shape.smemTile;
        stats->pairSh = p.pairSh != 0;
        stats->deepRegs = p.deepRegs != 0;
        stats->registers = shape.registers;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    cudaEventDestroy(eTuned);
}

// time grid of one object (FixedStep.h:7-37): step start epochs and sizes
static int buildGrid(double epochMjd, double duration, double step, int64_t maxSteps, std::vector<double>& t0,
                     std::vector<double>& dt, double& finalEt) {
    const double start = mjdToEtHost(epochMjd);
    const double end = mjdToEtHost(epochMjd + duration / 86400.0);
    const double span = end - start;
    if (!(span > 0) || !std::isfinite(span))
        throw std::runtime_error("Duration/step cannot be represented by the integration time/index types.");
    double cur = start, d = std::min(step, span);
    t0.clear();
    dt.clear();
    bool done = false;
    for (int64_t k = 0; k < maxSteps && !done; ++k) {
        t0.push_back(cur);
        dt.push_back(d);
        cur += d;
        const double rem = end - cur;
        done = rem <= 0;
        d = done ? 0 : std::min(step, rem);
    }
    finalEt = cur;
    return done ? 1 : 0;
}

void Engine::propagate(const TargetSet& t, int64_t maxSteps, const RunOptions& opt, std::vector<double>& outEpoch,
                       std::vector<double>& outState, RunStats* stats, cudaStream_t stream) {
    PHOP_CUDA(cudaSetDevice(device_));
    const int64_t n = (int64_t)t.size();
    if (n == 0) throw std::runtime_error("targets must be a nonempty array.");
    cudaEvent_t a0, a1;
    PHOP_CUDA(cudaEventCreate(&a0));
    PHOP_CUDA(cudaEventCreate(&a1));
    PHOP_CUDA(cudaEventRecord(a0, stream));
    std::vector<double> soa((size_t)6 * n), bc(n), ams(n);
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < 6; ++d) soa[(size_t)d * n + i] = t.state[(size_t)6 * i + d];
        // driver.cpp:118-120 then PrivateAccelerations.h:41-42
        const double area = t.dragArea[i] * 1e-6;
        const double crf = t.cr[i] * t.srpArea[i] / t.dragArea[i];
        ams[i] = crf * area / t.mass[i];
        bc[i] = t.cd[i] * area / t.mass[i];
    }
    double* dState = (double*)scratch("state", soa.size() * sizeof(double));
    double* dBc = (double*)scratch("bc", (size_t)n * sizeof(double));
    double* dAms = (double*)scratch("ams", (size_t)n * sizeof(double));
    PHOP_CUDA(cudaMemcpyAsync(dState, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
    PHOP_CUDA(cudaMemcpyAsync(dBc, bc.data(), bc.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
    PHOP_CUDA(cudaMemcpyAsync(dAms, ams.data(), ams.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
    bool uniform = true;
    for (int64_t i = 1; i < n && uniform; ++i)
        uniform = t.epoch[i] == t.epoch[0] && t.duration[i] == t.duration[0] && t.step[i] == t.step[0];
    outEpoch.assign(n, 0.0);
    RunStats local;
    RunStats* st = stats ? stats : &local;
    if (uniform) {
        std::vector<double> t0, dt;
        double finalEt = 0.0;
        if (!buildGrid(t.epoch[0], t.duration[0], t.step[0], maxSteps, t0, dt, finalEt))
            throw std::runtime_error("A target stopped without reaching the requested end of simulation.");
        TimeGrid g;
        g.shared = true;
        g.t0 = std::move(t0);
        g.dt = std::move(dt);
        int64_t launches = 0;
        const int64_t* dOrder = opt.ordered ? orderByRadius(n, dState, stream, &launches) : nullptr;
        runKernel(n, dState, dBc, dAms, g, dOrder, maxSteps, opt, st, stream, launches);
        std::fill(outEpoch.begin(), outEpoch.end(), etToMjdHost(finalEt));
        st->objectSteps += n * (int64_t)g.t0.size();
    } else {
        std::vector<double> cur(n), end(n), dtv(n), stp(n);
        std::vector<int64_t> cost(n), order(n);
        for (int64_t i = 0; i < n; ++i) {
            cur[i] = mjdToEtHost(t.epoch[i]);
            end[i] = mjdToEtHost(t.epoch[i] + t.duration[i] / 86400.0);
            const double span = end[i] - cur[i];
            if (!(span > 0) || !std::isfinite(span))
                throw std::runtime_error("Duration/step cannot be represented by the integration time/index types.");
            dtv[i] = std::min(t.step[i], span);
            stp[i] = t.step[i];
            cost[i] = (int64_t)std::ceil(span / t.step[i]);
            st->objectSteps += cost[i];
        }
        // longest objects first (in buckets of 2^(1/16) in step count), then
        // inside a bucket by geocentric radius (mixedOrder 0: warps take the
        // same drag-model branches), by start epoch (1: a warp's objects read
        // the same few epoch records), or drag / no drag and then epoch (2)
        std::vector<int> bucket(n), drag(n);
        std::vector<float> radius(n);
        const double dragR = host_.hasNrl ? (host_.shR > 0 ? host_.shR : 6378.137) + host_.nrlHcutoff + 200.0 : 0.0;
        for (int64_t i = 0; i < n; ++i) {
            bucket[i] = (int)std::floor(16.0 * std::log2((double)std::max<int64_t>(cost[i], 1)));
            const double* x = &t.state[(size_t)6 * i];
            radius[i] = (float)(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
            drag[i] = radius[i] < dragR * dragR ? 1 : 0;
        }
        std::iota(order.begin(), order.end(), 0);
        const int mode = opt.ordered ? opt.mixedOrder : -1;
        std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
            if (bucket[a] != bucket[b]) return bucket[a] > bucket[b];
            if (mode == 0) return radius[a] < radius[b];
            if (mode == 2 && drag[a] != drag[b]) return drag[a] > drag[b];
            if (mode >= 1) return cur[a] < cur[b];
            return false;
        });
        double lo = cur[0], hi = end[0];
        for (int64_t i = 1; i < n; ++i) {
            lo = std::min(lo, cur[i]);
            hi = std::max(hi, end[i]);
        }
        double* dCur = (double*)scratch("cur", (size_t)n * 8);
        double* dEnd = (double*)scratch("end", (size_t)n * 8);
        double* dDt = (double*)scratch("dtv", (size_t)n * 8);
        double* dStep = (double*)scratch("step", (size_t)n * 8);
        int* dUnf = (int*)scratch("unfinished", (size_t)n * 4);
        int64_t* dOrder = (int64_t*)scratch("order", (size_t)n * 8);
        PHOP_CUDA(cudaMemcpyAsync(dCur, cur.data(), n * 8, cudaMemcpyHostToDevice, stream));
        PHOP_CUDA(cudaMemcpyAsync(dEnd, end.data(), n * 8, cudaMemcpyHostToDevice, stream));
        PHOP_CUDA(cudaMemcpyAsync(dDt, dtv.data(), n * 8, cudaMemcpyHostToDevice, stream));
        PHOP_CUDA(cudaMemcpyAsync(dStep, stp.data(), n * 8, cudaMemcpyHostToDevice, stream));
        PHOP_CUDA(cudaMemcpyAsync(dOrder, order.data(), n * 8, cudaMemcpyHostToDevice, stream));
        TimeGrid g;
        g.shared = false;
        g.cur = dCur;
        g.end = dEnd;
        g.dt1 = dDt;
        g.step = dStep;
        g.unfinished = dUnf;
        int64_t launches = 0;
        buildRecordGrid(lo, hi, g, stream, &launches);
        runKernel(n, dState, dBc, dAms, g, dOrder, maxSteps, opt, st, stream, launches);
        std::vector<int> unf(n);
        PHOP_CUDA(cudaMemcpy(cur.data(), dCur, n * 8, cudaMemcpyDeviceToHost));
        PHOP_CUDA(cudaMemcpy(unf.data(), dUnf, n * 4, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < n; ++i) {
            if (unf[i]) throw std::runtime_error("A target stopped without reaching the requested end of simulation.");
            outEpoch[i] = etToMjdHost(cur[i]);
        }
    }
    PHOP_CUDA(cudaMemcpyAsync(soa.data(), dState, soa.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    PHOP_CUDA(cudaEventRecord(a1, stream));
    PHOP_CUDA(cudaEventSynchronize(a1));
    float ms = 0;
    cudaEventElapsedTime(&ms, a0, a1);
    st->totalMs += ms;
    cudaEventDestroy(a0);
    cudaEventDestroy(a1);
    outState.assign((size_t)6 * n, 0.0);
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < 6; ++d) outState[(size_t)6 * i + d] = soa[(size_t)d * n + i];
}

// Per-object time of a sliced batch: over the unfinished objects (step
// size > 0) the earliest epoch and the latest epoch the next `maxSteps`
// steps can reach, per block; the unfinished count and the steps they will
// take (min(maxSteps, ceil(remaining / step)) each) by atomics.
__global__ void objectSpanKernel(const double* __restrict__ cur, const double* __restrict__ end,
                                 const double* __restrict__ dt, const double* __restrict__ step, int64_t n,
                                 int64_t maxSteps, double* __restrict__ blockLo, double* __restrict__ blockHi,
                                 unsigned long long* __restrict__ counts) {
    __shared__ double sLo[256], sHi[256];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double lo = INFINITY, hi = -INFINITY;
    if (i < n && dt[i] > 0.0) {
        const double c = cur[i], e = end[i], h = step[i];
        const double steps = fmin((double)maxSteps, ceil((e - c) / h));
        lo = c;
        hi = fmin(e, c + steps * h);
        atomicAdd(&counts[0], 1ull);
        atomicAdd(&counts[1], (unsigned long long)steps);
    }
    sLo[threadIdx.x] = lo;
    sHi[threadIdx.x] = hi;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) {
            sLo[threadIdx.x] = fmin(sLo[threadIdx.x], sLo[threadIdx.x + k]);
            sHi[threadIdx.x] = fmax(sHi[threadIdx.x], sHi[threadIdx.x + k]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        blockLo[blockIdx.x] = sLo[0];
        blockHi[blockIdx.x] = sHi[0];
    }
}

int64_t Engine::advanceObjects(int64_t n, double* dState, double* dTime, const double* dBc, const double* dAms,
                               int64_t maxSteps, const RunOptions& opt, RunStats* stats, cudaStream_t stream) {
    PHOP_CUDA(cudaSetDevice(device_));
    if (maxSteps <= 0) throw std::runtime_error("max_steps must be positive.");
    double* cur = dTime;
    double* end = dTime + n;
    double* dtv = dTime + 2 * n;
    double* stp = dTime + 3 * n;
    RunStats local;
    RunStats* st = stats ? stats : &local;
    const int threads = 256;
    const int blocks = (int)((n + threads - 1) / threads);
    double* dLo = (double*)scratch("spanLo", (size_t)blocks * 8);
    double* dHi = (double*)scratch("spanHi", (size_t)blocks * 8);
    unsigned long long* dCounts = (unsigned long long*)scratch("spanCounts", 16);
    auto span = [&](double& lo, double& hi, int64_t& unfinished, int64_t& steps) {
        PHOP_CUDA(cudaMemsetAsync(dCounts, 0, 16, stream));
        objectSpanKernel<<<blocks, threads, 0, stream>>>(cur, end, dtv, stp, n, maxSteps, dLo, dHi, dCounts);
        PHOP_CUDA(cudaGetLastError());
        std::vector<double> l(blocks), h(blocks);
        unsigned long long c[2];
        PHOP_CUDA(cudaMemcpyAsync(l.data(), dLo, (size_t)blocks * 8, cudaMemcpyDeviceToHost, stream));
        PHOP_CUDA(cudaMemcpyAsync(h.data(), dHi, (size_t)blocks * 8, cudaMemcpyDeviceToHost, stream));
        PHOP_CUDA(cudaMemcpyAsync(c, dCounts, 16, cudaMemcpyDeviceToHost, stream));
        PHOP_CUDA(cudaStreamSynchronize(stream));
        lo = INFINITY;
        hi = -INFINITY;
        for (int b = 0; b < blocks; ++b) {
            lo = std::min(lo, l[b]);
            hi = std::max(hi, h[b]);
        }
        unfinished = (int64_t)c[0];
        steps = (int64_t)c[1];
    };
    double lo, hi;
    int64_t unfinished, steps;
    span(lo, hi, unfinished, steps);
    if (unfinished == 0) return 0;
    TimeGrid g;
    g.shared = false;
    g.cur = cur;
    g.end = end;
    g.dt1 = dtv;
    g.step = stp;
    g.unfinished = (int*)scratch("unfinished", (size_t)n * 4);
    int64_t launches = 1;  // the span kernel
    buildRecordGrid(lo, hi, g, stream, &launches);
    const int64_t* dOrder = opt.ordered ? orderByRadius(n, dState, stream, &launches) : nullptr;
    RunOptions o = opt;
    o.graph = false;  // every slice's launch parameters differ: nothing to replay
    runKernel(n, dState, dBc, dAms, g, dOrder, maxSteps, o, st, stream, launches);
    st->objectSteps += steps;
    span(lo, hi, unfinished, steps);
    st->launches += 1;
    return unfinished;
}

void Engine::propagateResident(int64_t n, double* dState, const double* epochMjd, const double* bc, const double* ams,
                               double duration, double step, int64_t maxSteps, const RunOptions& opt,
                               std::vector<double>& outEpochMjd, RunStats* stats, cudaStream_t stream) {
    PHOP_CUDA(cudaSetDevice(device_));
    for (int64_t i = 1; i < n; ++i)
        if (epochMjd[i] != epochMjd[0])
            throw std::runtime_error("The resident entry point needs one common epoch.");
    std::vector<double> t0, dt;
    double finalEt = 0;
    if (!buildGrid(epochMjd[0], duration, step, maxSteps, t0, dt, finalEt))
        throw std::runtime_error("A target stopped without reaching the requested end of simulation.");
    double* dBc = (double*)scratch("bc", (size_t)n * 8);
    double* dAms = (double*)scratch("ams", (size_t)n * 8);
    PHOP_CUDA(cudaMemcpyAsync(dBc, bc, (size_t)n * 8, cudaMemcpyHostToDevice, stream));
    PHOP_CUDA(cudaMemcpyAsync(dAms, ams, (size_t)n * 8, cudaMemcpyHostToDevice, stream));
    RunStats local;
    RunStats* st = stats ? stats : &local;
    const int64_t nsteps = (int64_t)t0.size();
    TimeGrid g;
    g.shared = true;
    g.t0 = std::move(t0);
    g.dt = std::move(dt);
    int64_t launches = 0;
    const int64_t* dOrder = opt.ordered ? orderByRadius(n, dState, stream, &launches) : nullptr;
    runKernel(n, dState, dBc, dAms, g, dOrder, maxSteps, opt, st, stream, launches);
    st->objectSteps += n * nsteps;
    outEpochMjd.assign(n, etToMjdHost(finalEt));
}

}  // namespace phop
