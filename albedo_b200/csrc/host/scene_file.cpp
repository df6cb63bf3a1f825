// Scene-file and OBJ reading for the reference's formats: the scene grammar of
// scene/scene_file.cpp (statements, value ranges, limits, mesh path rules,
// instance operations, messages) and the OBJ subset of geometry/obj.cpp (v / vt
// / f statements, fan triangulation, negative indices), with numbers parsed by
// std::from_chars as io/tokens.cpp:25-52 parses them. The scene grammar is
// table-driven (see "scene reading" below); large OBJ files are read in pieces
// on several threads.
#include "scene_file.hpp"

#include <algorithm>
#include <charconv>
#include <format>
#include <fstream>
#include <functional>
#include <map>
#include <optional>
#include <span>
#include <sstream>
#include <string_view>
#include <thread>
#include <variant>
#include <vector>

namespace albedo_b200 {

SceneParseError::SceneParseError(std::size_t line, const std::string& problem)
    : std::runtime_error{line == 0 ? std::format("scene: {}", problem) : std::format("scene line {}: {}", line, problem)},
      line_number{line}
{
}

namespace {

// Limits of scene/scene_file.hpp:17-37 and geometry/obj.hpp:16-28.
constexpr std::size_t kMaxSceneLine{4096};
constexpr std::size_t kMaxObjects{4096};
constexpr std::size_t kMaxMaterials{4096};
constexpr std::size_t kMaxMeshes{16};
constexpr std::size_t kMaxInstanceOperations{16};
constexpr std::size_t kMaxGroundPoints{std::size_t{1} << 26U};
constexpr std::size_t kMaxObjLine{65536};
constexpr std::size_t kObjBudget{std::size_t{1} << 24U};

// Value ranges, scene/scene_file.cpp:68-77.
constexpr double kMaxReflectance{1};
constexpr double kMaxEmission{1e6};
constexpr double kMaxRoughness{1};
constexpr double kMinIor{1e-2};
constexpr double kMaxIor{1e2};
constexpr double kMinConductorEta{1e-3};
constexpr double kMaxConductorEta{1e3};
constexpr double kMaxConductorK{1e3};
constexpr double kMaxPerlinVeins{1e2};

// Splits a line at runs of " \t\r\v\f" (io/tokens.cpp:12-23).
class Words {
public:
    explicit Words(std::string_view line) : rest{line} {}
    std::optional<std::string_view> next()
    {
        constexpr std::string_view blanks{" \t\r\v\f"};
        const std::size_t start{rest.find_first_not_of(blanks)};
        if (start == std::string_view::npos) {
            rest = {};
            return std::nullopt;
        }
        rest.remove_prefix(start);
        const std::size_t end{std::min(rest.find_first_of(blanks), rest.size())};
        const std::string_view word{rest.substr(0, end)};
        rest.remove_prefix(end);
        return word;
    }

private:
    std::string_view rest;
};

std::optional<double> parseReal(std::string_view token)
{
    if (token.starts_with('+')) {
        token.remove_prefix(1);
        if (token.starts_with('+') || token.starts_with('-')) {
            return std::nullopt;
        }
    }
    double value{};
    const auto [end, error]{std::from_chars(token.data(), token.data() + token.size(), value)};
    if (error != std::errc{} || end != token.data() + token.size() || !std::isfinite(value)) {
        return std::nullopt;
    }
    return value;
}

std::optional<long long> parseInteger(std::string_view token)
{
    long long value{};
    const auto [end, error]{std::from_chars(token.data(), token.data() + token.size(), value)};
    if (error != std::errc{} || end != token.data() + token.size() || token.empty()) {
        return std::nullopt;
    }
    return value;
}

// Reads lines terminated by '\n' (a trailing '\r' stays part of the line and is
// whitespace to the tokenizer), failing on lines longer than `limit`.
template <typename OnLine>
void forEachLine(std::istream& input, std::size_t limit, OnLine&& on_line,
                 const std::function<void(std::size_t)>& too_long)
{
    std::string line;
    std::size_t number{0};
    while (std::getline(input, line)) {
        ++number;
        if (line.size() > limit) {
            too_long(number);
        }
        on_line(std::string_view{line}, number);
    }
    if (input.bad()) {
        throw std::runtime_error{"reading failed"};
    }
}

bool isIdentifier(std::string_view name)
{
    const auto letter = [](char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z'); };
    const auto digit = [](char c) { return c >= '0' && c <= '9'; };
    if (name.empty() || (!letter(name.front()) && name.front() != '_')) {
        return false;
    }
    return std::ranges::all_of(name, [&](char c) { return letter(c) || digit(c) || c == '_' || c == '-'; });
}

// Quotes input for an error message: at most 32 bytes, non-printable bytes escaped.
std::string quoted(std::string_view token)
{
    std::string result{"'"};
    for (const char c : token.substr(0, 32)) {
        const auto byte{static_cast<unsigned char>(c)};
        if (byte >= 0x20 && byte <= 0x7E) {
            result += c;
        } else {
            result += std::format("\\x{:02X}", byte);
        }
    }
    result += token.size() > 32 ? "'..." : "'";
    return result;
}

// ---------------------------------------------------------------- OBJ reading

struct ObjMesh {
    std::vector<Vec3> positions;
    std::vector<std::array<double, 2>> uvs;
    std::vector<std::array<std::uint32_t, 3>> faces;
    std::vector<std::array<std::uint32_t, 3>> texture_faces;
};

struct ObjBudget {
    std::size_t vertices{kObjBudget};
    std::size_t texture_coordinates{kObjBudget};
    std::size_t triangles{kObjBudget};
};

class ObjError : public std::runtime_error {
public:
    ObjError(std::size_t line, const std::string& problem)
        : std::runtime_error{std::format("OBJ line {}: {}", line, problem)}
    {
    }
    // The same error again, from its full message.
    static ObjError fromMessage(const std::string& message) { return ObjError{message}; }

private:
    explicit ObjError(const std::string& message) : std::runtime_error{message} {}
};

// Calls on_line(line, index) for every line of `text` as std::getline splits
// it: at each '\n', plus a last line when the text does not end with one.
template <typename OnLine>
void forEachTextLine(std::string_view text, OnLine&& on_line)
{
    std::size_t index{0};
    std::size_t begin{0};
    while (begin < text.size()) {
        const std::size_t end{text.find('\n', begin)};
        if (end == std::string_view::npos) {
            on_line(text.substr(begin), index);
            return;
        }
        on_line(text.substr(begin, end - begin), index++);
        begin = end + 1;
    }
}

// A piece of an OBJ text made of whole lines, with what its lines define. The
// pieces of a large file are read on separate threads: a first pass counts each
// piece's lines, vertices, texture coordinates and triangles, which gives every
// piece the counts of all lines before it, and a second pass reads each piece
// with those counts as if the lines before it had just been read. The pieces'
// results are joined in order, and the error of the earliest failing line is the
// one reported, so the result is the one-thread reader's, error messages
// included.
struct ObjPiece {
    std::string_view text;
    std::size_t lines{0};
    std::size_t positions{0};
    std::size_t uvs{0};
    std::size_t triangles{0};
};

struct ObjPieceResult {
    ObjMesh mesh;
    bool every_face_textured{true};
    std::size_t error_line{0};  // 0: no error
    std::string error;
};

void countObjPiece(ObjPiece& piece)
{
    forEachTextLine(piece.text, [&](std::string_view line, std::size_t) {
        ++piece.lines;
        Words words{line.substr(0, line.find('#'))};
        const auto keyword{words.next()};
        if (keyword == "v") {
            ++piece.positions;
        } else if (keyword == "vt") {
            ++piece.uvs;
        } else if (keyword == "f") {
            std::size_t corners{0};
            while (words.next()) {
                ++corners;
            }
            piece.triangles += corners >= 3 ? corners - 2 : 0;
        }
    });
}

// Reads one piece (geometry/obj.cpp's per-line rules) whose first line has
// number `first_line` and follows `before` (the counts of all earlier lines).
// Stops at the piece's first error and records it.
void readObjPiece(std::string_view text, std::size_t first_line, const ObjPiece& before, const ObjBudget& budget,
                  ObjPieceResult& out)
{
    ObjMesh& mesh{out.mesh};
    struct Corner {
        std::uint32_t position{};
        std::optional<std::uint32_t> texture;
    };
    std::vector<Corner> corners;
    std::size_t line_number{0};
    auto fail = [&](const std::string& problem) -> void { throw ObjError{line_number, problem}; };
    auto number = [&](std::string_view token) {
        const auto value{parseReal(token)};
        if (!value) {
            fail("a coordinate is not a finite number");
        }
        return *value;
    };
    auto resolved = [&](long long index, std::string_view kind, std::size_t count) -> std::uint32_t {
        if (index > 0) {
            if (static_cast<unsigned long long>(index) > count) {
                fail(std::format("a face refers to a {} not yet defined", kind));
            }
            return static_cast<std::uint32_t>(index - 1);
        }
        if (index < 0) {
            const auto back{static_cast<unsigned long long>(-(index + 1)) + 1};
            if (back > count) {
                fail(std::format("a face refers to a {} before the first one", kind));
            }
            return static_cast<std::uint32_t>(count - back);
        }
        fail("a face uses index 0; OBJ indices start at 1");
        return 0;
    };
    auto optional_index = [&](std::string_view part) -> std::optional<long long> {
        if (part.empty()) {
            return std::nullopt;
        }
        const auto index{parseInteger(part)};
        if (!index) {
            fail("a face corner is not a valid index");
        }
        return index;
    };
    try {
        forEachTextLine(text, [&](std::string_view line, std::size_t index) {
            line_number = first_line + index;
            if (line.size() > kMaxObjLine) {
                fail(std::format("line longer than {} bytes", kMaxObjLine));
            }
            Words words{line.substr(0, line.find('#'))};
            const auto keyword{words.next()};
            if (keyword == "v") {
                if (before.positions + mesh.positions.size() >= budget.vertices) {
                    fail(std::format("more than {} vertices", budget.vertices));
                }
                std::array<double, 3> xyz{};
                for (double& c : xyz) {
                    const auto token{words.next()};
                    if (!token) {
                        fail("a vertex needs three coordinates");
                    }
                    c = number(*token);
                }
                while (const auto extra{words.next()}) {
                    static_cast<void>(number(*extra));
                }
                mesh.positions.push_back({xyz[0], xyz[1], xyz[2]});
            } else if (keyword == "vt") {
                if (before.uvs + mesh.uvs.size() >= budget.texture_coordinates) {
                    fail(std::format("more than {} texture coordinates", budget.texture_coordinates));
                }
                const auto u{words.next()};
                if (!u) {
                    fail("a texture coordinate needs at least u");
                }
                std::array<double, 2> uv{number(*u), 0.0};
                if (const auto v{words.next()}) {
                    uv[1] = number(*v);
                }
                while (const auto extra{words.next()}) {
                    static_cast<void>(number(*extra));
                }
                mesh.uvs.push_back(uv);
            } else if (keyword == "f") {
                corners.clear();
                const std::size_t positions{before.positions + mesh.positions.size()};
                const std::size_t uvs{before.uvs + mesh.uvs.size()};
                while (const auto token{words.next()}) {
                    const std::size_t slash{token->find('/')};
                    const auto position{parseInteger(token->substr(0, slash))};
                    if (!position) {
                        fail("a face corner is not a valid index");
                    }
                    Corner corner{resolved(*position, "vertex", positions), std::nullopt};
                    if (slash != std::string_view::npos) {
                        const std::string_view rest{token->substr(slash + 1)};
                        const std::size_t second{rest.find('/')};
                        if (const auto texture{optional_index(rest.substr(0, second))}) {
                            corner.texture = resolved(*texture, "texture coordinate", uvs);
                        }
                        if (second != std::string_view::npos) {
                            static_cast<void>(optional_index(rest.substr(second + 1)));
                        }
                    }
                    corners.push_back(corner);
                }
                if (corners.size() < 3) {
                    fail("a face needs at least three corners");
                }
                if (corners.size() - 2 > budget.triangles - (before.triangles + mesh.faces.size())) {
                    fail(std::format("more than {} triangles", budget.triangles));
                }
                for (std::size_t c{1}; c + 1 < corners.size(); ++c) {
                    const Corner& a{corners[0]};
                    const Corner& b{corners[c]};
                    const Corner& d{corners[c + 1]};
                    mesh.faces.push_back({a.position, b.position, d.position});
                    if (!a.texture || !b.texture || !d.texture) {
                        out.every_face_textured = false;
                        mesh.texture_faces.clear();
                    } else if (out.every_face_textured) {
                        mesh.texture_faces.push_back({*a.texture, *b.texture, *d.texture});
                    }
                }
            }
        });
    } catch (const ObjError& error) {
        out.error_line = line_number;
        out.error = error.what();
    }
}

// Pieces of at least this many bytes are worth a thread of their own.
constexpr std::size_t kObjPieceBytes{std::size_t{1} << 20U};

// geometry/obj.cpp's reader over text in memory, in `pieces` pieces (1: one
// thread); the result does not depend on the number of pieces.
ObjMesh parseObj(std::string_view text, const ObjBudget& budget, unsigned pieces)
{
    // Split at line ends near equal byte offsets.
    std::vector<ObjPiece> parts;
    std::size_t begin{0};
    for (unsigned k{1}; k <= pieces && begin < text.size(); ++k) {
        std::size_t end{k == pieces ? text.size() : text.size() / pieces * k};
        if (end < begin) {
            end = begin;
        }
        if (end < text.size()) {
            const std::size_t newline{text.find('\n', end == 0 ? 0 : end - 1)};
            end = newline == std::string_view::npos ? text.size() : newline + 1;
        }
        if (end > begin) {
            parts.push_back({.text = text.substr(begin, end - begin)});
            begin = end;
        }
    }
    const auto onThreads = [&](auto&& work) {
        // A jthread joins when destroyed, so an exception that leaves early (a
        // thread that fails to start, or the calling thread's own share) still
        // waits for the workers already running.
        std::vector<std::jthread> workers;
        for (std::size_t k{1}; k < parts.size(); ++k) {
            workers.emplace_back([&, k] { work(k); });
        }
        if (!parts.empty()) {
            work(0);
        }
        for (std::jthread& worker : workers) {
            worker.join();
        }
    };
    if (parts.size() > 1) {
        onThreads([&](std::size_t k) { countObjPiece(parts[k]); });
    }
    // The counts of all lines before each piece.
    std::vector<ObjPiece> before(parts.size());
    for (std::size_t k{1}; k < parts.size(); ++k) {
        before[k] = {.lines = before[k - 1].lines + parts[k - 1].lines,
                     .positions = before[k - 1].positions + parts[k - 1].positions,
                     .uvs = before[k - 1].uvs + parts[k - 1].uvs,
                     .triangles = before[k - 1].triangles + parts[k - 1].triangles};
    }
    std::vector<ObjPieceResult> results(parts.size());
    std::vector<std::exception_ptr> failures(parts.size());
    onThreads([&](std::size_t k) {
        try {
            readObjPiece(parts[k].text, before[k].lines + 1, before[k], budget, results[k]);
        } catch (...) {
            failures[k] = std::current_exception();
        }
    });
    // The earliest failure in file order is the one the one-thread reader meets.
    for (std::size_t k{0}; k < parts.size(); ++k) {
        if (failures[k]) {
            std::rethrow_exception(failures[k]);
        }
        if (results[k].error_line != 0) {
            throw ObjError::fromMessage(results[k].error);
        }
    }
    if (results.size() == 1) {
        ObjMesh mesh{std::move(results[0].mesh)};
        if (!results[0].every_face_textured) {
            mesh.texture_faces.clear();
        }
        return mesh;
    }
    ObjMesh mesh;
    bool every_face_textured{true};
    std::size_t positions{0}, uvs{0}, faces{0};
    for (const ObjPieceResult& r : results) {
        positions += r.mesh.positions.size();
        uvs += r.mesh.uvs.size();
        faces += r.mesh.faces.size();
        every_face_textured = every_face_textured && r.every_face_textured;
    }
    mesh.positions.reserve(positions);
    mesh.uvs.reserve(uvs);
    mesh.faces.reserve(faces);
    for (const ObjPieceResult& r : results) {
        mesh.positions.insert(mesh.positions.end(), r.mesh.positions.begin(), r.mesh.positions.end());
        mesh.uvs.insert(mesh.uvs.end(), r.mesh.uvs.begin(), r.mesh.uvs.end());
        mesh.faces.insert(mesh.faces.end(), r.mesh.faces.begin(), r.mesh.faces.end());
    }
    if (every_face_textured) {
        mesh.texture_faces.reserve(faces);
        for (const ObjPieceResult& r : results) {
            mesh.texture_faces.insert(mesh.texture_faces.end(), r.mesh.texture_faces.begin(),
                                      r.mesh.texture_faces.end());
        }
    }
    return mesh;
}

ObjMesh readObj(const std::filesystem::path& path, const ObjBudget& budget)
{
    std::ifstream file{path, std::ios::binary};
    if (!file) {
        throw std::runtime_error{"cannot open OBJ file"};
    }
    std::string text;
    std::array<char, 1 << 16> block{};
    while (file.read(block.data(), static_cast<std::streamsize>(block.size())) || file.gcount() > 0) {
        text.append(block.data(), static_cast<std::size_t>(file.gcount()));
        if (file.eof()) {
            break;
        }
    }
    if (file.bad()) {
        throw std::runtime_error{"reading failed"};
    }
    const unsigned threads{std::max(1u, std::thread::hardware_concurrency())};
    const auto pieces{static_cast<unsigned>(std::clamp<std::size_t>(text.size() / kObjPieceBytes, 1, threads))};
    return parseObj(text, budget, pieces);
}

// ---------------------------------------------------------------- scene reading
//
// The scene grammar is held as data. A statement is a keyword, a few positional
// values and a set of named fields, given in any order, each at most once. Every
// value has a kind (a number, a positive number, a number in a range, a point, a
// colour whose channels lie in a range, a material name), the noun its error
// messages use, and its range. One loop reads the named fields of any statement
// against its table and one function reads a value of any kind; a short builder
// per statement then turns the values into scene content and checks what a table
// cannot say: which fields are required (reported in the builder's order),
// camera and sphere validity, mesh files and instance placement. The limits,
// ranges and messages are the reference's (scene/scene_file.cpp:17-77 and its
// statement readers), so a file is accepted or refused, with the same words, by
// both readers.

// One line's words, read front to back; every error names the line.
class LineWords {
public:
    LineWords(std::string_view text, std::size_t line) : number{line}
    {
        Words split{text};
        while (const auto word{split.next()}) {
            words.push_back(*word);
        }
    }

    [[noreturn]] void fail(const std::string& problem) const { throw SceneParseError{number, problem}; }

    bool done() const { return at == words.size(); }
    std::optional<std::string_view> peek() const
    {
        return done() ? std::nullopt : std::optional<std::string_view>{words[at]};
    }
    std::optional<std::string_view> take()
    {
        return done() ? std::nullopt : std::optional<std::string_view>{words[at++]};
    }
    // The next word, which must exist; `noun` names it when it does not.
    std::string_view expect(std::string_view noun)
    {
        if (done()) {
            fail(std::format("expected {}", noun));
        }
        return words[at++];
    }
    void end() const
    {
        if (!done()) {
            fail(std::format("unexpected {}", quoted(words[at])));
        }
    }

private:
    std::vector<std::string_view> words;
    std::size_t at{0};
    std::size_t number;
};

enum class Kind : std::uint8_t {
    Number,   // any finite number
    Positive, // a number above zero
    Ranged,   // a number in [low, high]
    Point,    // three numbers: the x, y and z coordinates of <noun>
    Color,    // three numbers in [low, high]: the red, green and blue channels of <noun>
    Material, // the name of a defined material
    Basic,    // the name of a defined material that is not a mix
};

struct Field {
    std::string_view key;
    Kind kind;
    std::string_view noun;
    double low{0};
    double high{0};
};

using Value = std::variant<double, Vec3, Rgb, std::uint32_t>;

constexpr double kAnyNumber{0};

// Value ranges (scene/scene_file.cpp:68-77) as the field tables use them.
constexpr Field reflectance(std::string_view key, std::string_view noun)
{
    return {key, Kind::Color, noun, 0, kMaxReflectance};
}
constexpr Field emission(std::string_view key, std::string_view noun)
{
    return {key, Kind::Color, noun, 0, kMaxEmission};
}

constexpr std::array kCameraFields{
    Field{"from", Kind::Point, "the camera position"},
    Field{"at", Kind::Point, "the point the camera looks at"},
    Field{"up", Kind::Point, "the camera's up direction"},
    Field{"fov", Kind::Number, "the field of view"},
};
constexpr std::array kSkyFields{
    emission("nadir", "the radiance from below"),
    emission("zenith", "the radiance from above"),
};
constexpr std::array kDiffuseFields{reflectance("color", "the color")};
constexpr std::array kCheckerFields{
    reflectance("even", "the even color"),
    reflectance("odd", "the odd color"),
    Field{"frequency", Kind::Positive, "the checker frequency"},
};
constexpr std::array kPerlinFields{
    reflectance("low", "the low color"),
    reflectance("high", "the high color"),
    Field{"scale", Kind::Positive, "the noise scale"},
    Field{"veins", Kind::Ranged, "the veins", 0, kMaxPerlinVeins},
};
constexpr std::array kConductorFields{
    Field{"eta", Kind::Color, "the refractive index", kMinConductorEta, kMaxConductorEta},
    Field{"k", Kind::Color, "the absorption", 0, kMaxConductorK},
    Field{"roughness", Kind::Ranged, "the roughness", 0, kMaxRoughness},
};
constexpr std::array kDielectricFields{
    Field{"ior", Kind::Ranged, "the index of refraction", kMinIor, kMaxIor},
    Field{"roughness", Kind::Ranged, "the roughness", 0, kMaxRoughness},
};
constexpr std::array kMixFields{
    Field{"first", Kind::Basic, "a material name"},
    Field{"second", Kind::Basic, "a material name"},
    Field{"scale", Kind::Positive, "the noise scale"},
    Field{"veins", Kind::Ranged, "the veins", 0, kMaxPerlinVeins},
    Field{"threshold", Kind::Ranged, "the threshold", 0, 1},
};
constexpr std::array kSphereFields{
    Field{"radius", Kind::Number, "a radius"},
    Field{"material", Kind::Material, "a material name"},
};
constexpr std::array kPointLightFields{emission("intensity", "the intensity")};
constexpr std::array kAreaLightFields{
    Field{"radius", Kind::Number, "a radius"},
    emission("radiance", "the radiance"),
    Field{"material", Kind::Material, "a material name"},
};

double readNumber(LineWords& line, std::string_view noun)
{
    const std::string_view token{line.expect(noun)};
    const auto value{parseReal(token)};
    if (!value) {
        line.fail(std::format("{} must be a finite number, got {}", noun, quoted(token)));
    }
    return *value;
}

// One number of kind Number, Positive or Ranged, checked as soon as it is read.
double readScalar(LineWords& line, Kind kind, std::string_view noun, double low, double high)
{
    const double value{readNumber(line, noun)};
    if (kind == Kind::Positive && !(value > 0)) {
        line.fail(std::format("{} must be positive, got {}", noun, value));
    }
    if (kind == Kind::Ranged && (value < low || value > high)) {
        line.fail(std::format("{} must be between {} and {}, got {}", noun, low, high, value));
    }
    return value;
}

// A point (three numbers) or a colour (three numbers in [low, high]).
std::array<double, 3> readTriple(LineWords& line, Kind kind, std::string_view noun, double low = kAnyNumber,
                                 double high = kAnyNumber)
{
    static constexpr std::array<std::string_view, 3> kCoordinates{"x coordinate", "y coordinate", "z coordinate"};
    static constexpr std::array<std::string_view, 3> kChannels{"red channel", "green channel", "blue channel"};
    const bool color{kind == Kind::Color};
    std::array<double, 3> out{};
    for (std::size_t k{0}; k < 3; ++k) {
        const std::string part{std::format("the {} of {}", color ? kChannels[k] : kCoordinates[k], noun)};
        out[k] = readScalar(line, color ? Kind::Ranged : Kind::Number, part, low, high);
    }
    return out;
}

Vec3 readPoint(LineWords& line, std::string_view noun)
{
    const auto v{readTriple(line, Kind::Point, noun)};
    return {v[0], v[1], v[2]};
}

Rgb readColor(LineWords& line, std::string_view noun, double low, double high)
{
    const auto v{readTriple(line, Kind::Color, noun, low, high)};
    return {v[0], v[1], v[2]};
}

std::string_view readName(LineWords& line, std::string_view noun)
{
    const std::string_view token{line.expect(noun)};
    if (!isIdentifier(token)) {
        line.fail(std::format("{} is not a valid name", quoted(token)));
    }
    return token;
}

// Named values read from one statement, in the slots of its field table.
class FieldValues {
public:
    explicit FieldValues(std::span<const Field> fields) : table{fields}, values(fields.size()) {}

    std::optional<std::size_t> slot(std::string_view key) const
    {
        for (std::size_t i{0}; i < table.size(); ++i) {
            if (table[i].key == key) {
                return i;
            }
        }
        return std::nullopt;
    }
    bool given(std::size_t i) const { return values[i].has_value(); }
    void set(std::size_t i, Value value) { values[i] = value; }

    template <typename T>
    std::optional<T> get(std::string_view key) const
    {
        const auto& value{values[*slot(key)]};
        return value ? std::optional<T>{std::get<T>(*value)} : std::nullopt;
    }
    // A required field: its absence is the statement's error.
    template <typename T>
    T need(const LineWords& line, std::string_view key) const
    {
        const auto value{get<T>(key)};
        if (!value) {
            line.fail(std::format("missing '{}'", key));
        }
        return *value;
    }

private:
    std::span<const Field> table;
    std::vector<std::optional<Value>> values;
};

struct MeshEntry {
    std::uint32_t id{};
    std::vector<Vec3> points; // positions that kept triangles use, each once
};

// Everything a scene file has defined so far.
struct SceneState {
    std::filesystem::path directory;
    HostScene scene;
    bool sky_given{false};
    std::map<std::string, std::uint32_t, std::less<>> material_ids;
    std::map<std::string, MeshEntry, std::less<>> meshes;
    ObjBudget budget{};
    std::size_t ground_points_left{kMaxGroundPoints};
    std::size_t objects{0};

    std::uint32_t materialNamed(LineWords& line) const
    {
        const std::string_view name{readName(line, "a material name")};
        const auto found{material_ids.find(name)};
        if (found == material_ids.end()) {
            line.fail(std::format("material {} is not defined", quoted(name)));
        }
        return found->second;
    }

    void countObject(const LineWords& line)
    {
        if (objects >= kMaxObjects) {
            line.fail(std::format("more than {} objects", kMaxObjects));
        }
        ++objects;
    }
};

Value readValue(LineWords& line, const Field& field, const SceneState& state)
{
    switch (field.kind) {
    case Kind::Point:
        return readPoint(line, field.noun);
    case Kind::Color:
        return readColor(line, field.noun, field.low, field.high);
    case Kind::Material:
        return state.materialNamed(line);
    case Kind::Basic: {
        const std::string_view name{line.peek().value_or("")};
        const std::uint32_t id{state.materialNamed(line)};
        if (state.scene.materials[id].mix) {
            line.fail(std::format("material {} is a mix, and a mix cannot hold another mix", quoted(name)));
        }
        return id;
    }
    default:
        return readScalar(line, field.kind, field.noun, field.low, field.high);
    }
}

// The generic field loop: the rest of the line is key / value pairs from `table`.
FieldValues readFields(LineWords& line, std::span<const Field> table, const SceneState& state)
{
    FieldValues values{table};
    while (const auto key{line.take()}) {
        const auto slot{values.slot(*key)};
        if (slot && values.given(*slot)) {
            line.fail(std::format("{} is given twice", quoted(*key)));
        }
        if (!slot) {
            line.fail(std::format("unknown field {}", quoted(*key)));
        }
        values.set(*slot, readValue(line, table[*slot], state));
    }
    return values;
}

// ------------------------------------------------ materials

struct MaterialType {
    std::string_view name;
    std::span<const Field> fields;
    MaterialDesc (*build)(const FieldValues&, const LineWords&, const SceneState&);
};

MaterialDesc diffuseMaterial(const FieldValues& f, const LineWords& line, const SceneState&)
{
    MaterialDesc m;
    m.first.texture = {TextureKind::Constant, f.need<Rgb>(line, "color")};
    return m;
}

MaterialDesc checkerMaterial(const FieldValues& f, const LineWords& line, const SceneState&)
{
    MaterialDesc m;
    const Rgb even{f.need<Rgb>(line, "even")};
    const Rgb odd{f.need<Rgb>(line, "odd")};
    m.first.texture = {TextureKind::Checker, even, odd, f.need<double>(line, "frequency")};
    return m;
}

MaterialDesc perlinMaterial(const FieldValues& f, const LineWords& line, const SceneState&)
{
    MaterialDesc m;
    const Rgb low{f.need<Rgb>(line, "low")};
    const Rgb high{f.need<Rgb>(line, "high")};
    const double scale{f.need<double>(line, "scale")};
    m.first.texture = {TextureKind::Perlin, low, high, scale, f.get<double>("veins").value_or(0)};
    return m;
}

MaterialDesc conductorMaterial(const FieldValues& f, const LineWords& line, const SceneState&)
{
    MaterialDesc m;
    m.first.kind = BasicKind::Conductor;
    m.first.eta = f.need<Rgb>(line, "eta");
    m.first.k = f.need<Rgb>(line, "k");
    m.first.roughness = f.get<double>("roughness").value_or(0);
    const std::array<double, 3> eta{m.first.eta.r, m.first.eta.g, m.first.eta.b};
    const std::array<double, 3> k{m.first.k.r, m.first.k.g, m.first.k.b};
    for (std::size_t c{0}; c < 3; ++c) {
        // Such a channel reflects nothing: the Fresnel term is 0/0.
        if (eta[c] == 1 && k[c] == 0) {
            line.fail("a conductor channel cannot have eta 1 and k 0");
        }
    }
    return m;
}

MaterialDesc dielectricMaterial(const FieldValues& f, const LineWords& line, const SceneState&)
{
    MaterialDesc m;
    m.first.kind = BasicKind::Dielectric;
    m.first.ior = f.need<double>(line, "ior");
    m.first.roughness = f.get<double>("roughness").value_or(0);
    return m;
}

MaterialDesc mixMaterial(const FieldValues& f, const LineWords& line, const SceneState& state)
{
    MaterialDesc m;
    m.mix = true;
    m.first = state.scene.materials[f.need<std::uint32_t>(line, "first")].first;
    m.second = state.scene.materials[f.need<std::uint32_t>(line, "second")].first;
    m.scale = f.need<double>(line, "scale");
    m.veins = f.get<double>("veins").value_or(0);
    m.threshold = f.get<double>("threshold").value_or(0.5);
    return m;
}

constexpr std::array kMaterialTypes{
    MaterialType{"diffuse", kDiffuseFields, &diffuseMaterial},
    MaterialType{"checker", kCheckerFields, &checkerMaterial},
    MaterialType{"perlin", kPerlinFields, &perlinMaterial},
    MaterialType{"conductor", kConductorFields, &conductorMaterial},
    MaterialType{"dielectric", kDielectricFields, &dielectricMaterial},
    MaterialType{"mix", kMixFields, &mixMaterial},
};

// ------------------------------------------------ statements

void cameraStatement(SceneState& state, LineWords& line)
{
    if (state.scene.has_camera) {
        line.fail("the scene already has a camera");
    }
    const FieldValues f{readFields(line, kCameraFields, state)};
    CameraSettings settings{};
    settings.look_from = f.need<Vec3>(line, "from");
    settings.look_at = f.need<Vec3>(line, "at");
    settings.up = f.get<Vec3>("up").value_or(settings.up);
    settings.vertical_fov_degrees = f.get<double>("fov").value_or(settings.vertical_fov_degrees);
    try {
        static_cast<void>(buildCameraFrame(settings, 16.0 / 9.0));
    } catch (const std::invalid_argument& error) {
        line.fail(error.what());
    }
    state.scene.camera = settings;
    state.scene.has_camera = true;
}

void skyStatement(SceneState& state, LineWords& line)
{
    if (state.sky_given) {
        line.fail("the scene already has a sky");
    }
    const auto first{line.peek()};
    if (first && (*first == "nadir" || *first == "zenith")) {
        const FieldValues f{readFields(line, kSkyFields, state)};
        const Rgb nadir{f.need<Rgb>(line, "nadir")};
        state.scene.setSky(nadir, f.need<Rgb>(line, "zenith"));
    } else {
        // One radiance for the whole sky.
        const Rgb radiance{readColor(line, "the sky's radiance", 0, kMaxEmission)};
        line.end();
        state.scene.setSky(radiance, radiance);
    }
    state.sky_given = true;
}

void materialStatement(SceneState& state, LineWords& line)
{
    if (state.material_ids.size() >= kMaxMaterials) {
        line.fail(std::format("more than {} materials", kMaxMaterials));
    }
    const std::string_view name{readName(line, "a material name")};
    if (state.material_ids.contains(name)) {
        line.fail(std::format("material {} is already defined", quoted(name)));
    }
    const std::string_view type{line.expect("a material type")};
    const auto found{std::ranges::find(kMaterialTypes, type, &MaterialType::name)};
    if (found == kMaterialTypes.end()) {
        line.fail(std::format("unknown material type {}", quoted(type)));
    }
    const FieldValues f{readFields(line, found->fields, state)};
    const MaterialDesc material{found->build(f, line, state)};
    state.material_ids.emplace(std::string{name}, state.scene.addMaterial(material));
}

void checkSphere(const LineWords& line, Vec3 center, double radius)
{
    try {
        validateSphere(center, radius);
    } catch (const std::invalid_argument& error) {
        line.fail(error.what());
    }
}

void sphereStatement(SceneState& state, LineWords& line)
{
    state.countObject(line);
    const Vec3 center{readPoint(line, "the sphere center")};
    const FieldValues f{readFields(line, kSphereFields, state)};
    const double radius{f.need<double>(line, "radius")};
    checkSphere(line, center, radius);
    state.scene.addSphere(center, radius, f.need<std::uint32_t>(line, "material"));
}

void pointLightStatement(SceneState& state, LineWords& line)
{
    state.countObject(line);
    const Vec3 position{readPoint(line, "the light position")};
    const FieldValues f{readFields(line, kPointLightFields, state)};
    state.scene.addPointLight(position, f.need<Rgb>(line, "intensity"));
}

void areaLightStatement(SceneState& state, LineWords& line)
{
    state.countObject(line);
    const Vec3 center{readPoint(line, "the light center")};
    const FieldValues f{readFields(line, kAreaLightFields, state)};
    const double radius{f.need<double>(line, "radius")};
    checkSphere(line, center, radius);
    const Rgb radiance{f.need<Rgb>(line, "radiance")};
    // Without a material the light's sphere is black diffuse (scene/scene_file.cpp:819).
    std::optional<std::uint32_t> material{f.get<std::uint32_t>("material")};
    if (!material) {
        material = state.scene.addMaterial(MaterialDesc{});
    }
    state.scene.addAreaLight(center, radius, radiance, *material);
}

// Where a mesh statement's file lies. The path must be relative, without '..',
// control bytes or a root, and lead to a regular file inside the scene's
// directory (scene/scene_file.cpp:368-430 states the same rules).
std::filesystem::path meshFile(const LineWords& line, const std::filesystem::path& directory, std::string_view text)
{
    for (const char c : text) {
        const auto byte{static_cast<unsigned char>(c)};
        if (byte < 0x20 || byte == 0x7F) {
            line.fail(std::format("mesh path {} must be UTF-8 without control characters", quoted(text)));
        }
    }
    const std::filesystem::path relative{std::string{text}};
    const bool climbs{std::ranges::find(relative, std::filesystem::path{".."}) != relative.end()};
    if (relative.is_absolute() || relative.has_root_name() || relative.has_root_directory() || climbs) {
        line.fail(std::format("mesh path {} must be relative to the scene and not use '..'", quoted(text)));
    }
    std::error_code error;
    const std::filesystem::path base{std::filesystem::canonical(directory, error)};
    if (error) {
        line.fail("the scene's directory cannot be resolved");
    }
    const std::filesystem::path file{std::filesystem::weakly_canonical(base / relative, error)};
    if (error) {
        line.fail(std::format("cannot resolve mesh path {}", quoted(text)));
    }
    if (std::ranges::mismatch(base, file).in1 != base.end()) {
        line.fail(std::format("mesh path {} leads outside the scene's directory", quoted(text)));
    }
    switch (std::filesystem::status(file, error).type()) {
    case std::filesystem::file_type::regular:
        return file;
    case std::filesystem::file_type::not_found:
        line.fail(std::format("mesh file {} does not exist", quoted(text)));
    default:
        line.fail(std::format("mesh path {} is not a regular file", quoted(text)));
    }
}

// The positions that the mesh's kept triangles use, each once, in order: the
// points 'ground' examines.
std::vector<Vec3> usedPositions(const ObjMesh& obj)
{
    std::vector<bool> used(obj.positions.size(), false);
    for (const auto& f : obj.faces) {
        if (formsTriangle(obj.positions[f[0]], obj.positions[f[1]], obj.positions[f[2]])) {
            used[f[0]] = used[f[1]] = used[f[2]] = true;
        }
    }
    std::vector<Vec3> points;
    for (std::size_t i{0}; i < obj.positions.size(); ++i) {
        if (used[i]) {
            points.push_back(obj.positions[i]);
        }
    }
    return points;
}

void meshStatement(SceneState& state, LineWords& line)
{
    if (state.directory.empty()) {
        line.fail("meshes can only be read from a scene file, which they sit beside");
    }
    if (state.meshes.size() >= kMaxMeshes) {
        line.fail(std::format("more than {} meshes", kMaxMeshes));
    }
    const std::string_view name{readName(line, "a mesh name")};
    if (state.meshes.contains(name)) {
        line.fail(std::format("mesh {} is already defined", quoted(name)));
    }
    const std::string_view path{line.expect("a mesh file")};
    const bool smooth{line.peek() == "smooth"};
    if (smooth) {
        static_cast<void>(line.take());
    }
    line.end();
    const std::filesystem::path file{meshFile(line, state.directory, path)};
    ObjMesh obj;
    try {
        obj = readObj(file, state.budget);
    } catch (const ObjError& error) {
        line.fail(std::format("mesh {}: {}", quoted(path), error.what()));
    } catch (const std::runtime_error&) {
        line.fail(std::format("cannot read mesh file {}", quoted(path)));
    }
    MeshEntry entry{.id = 0, .points = usedPositions(obj)};
    if (entry.points.empty()) {
        line.fail(std::format("mesh {} has no triangles", quoted(path)));
    }
    try {
        entry.id = state.scene.addMesh(obj.positions, obj.faces, obj.uvs, obj.texture_faces, smooth);
    } catch (const std::exception& error) {
        line.fail(std::format("mesh {}: {}", quoted(path), error.what()));
    }
    state.budget.vertices -= obj.positions.size();
    state.budget.texture_coordinates -= obj.uvs.size();
    state.budget.triangles -= obj.faces.size();
    state.meshes.emplace(std::string{name}, std::move(entry));
}

// ------------------------------------------------ instance placement
//
// An instance's words after the mesh name are 'material <name>' once and up to
// kMaxInstanceOperations placement operations, each applied after the ones
// before it (scene/scene_file.cpp:962-1038 defines them).

using Operation = Transform (*)(SceneState&, LineWords&, const MeshEntry&, const Transform&);

Transform translateOperation(SceneState&, LineWords& line, const MeshEntry&, const Transform& placement)
{
    return Transform::translation(readPoint(line, "the translation")) * placement;
}

bool startsInstanceWord(std::string_view word);

// 'scale s' or 'scale sx sy sz': one factor when the next word is missing or
// starts the next operation.
Transform scaleOperation(SceneState&, LineWords& line, const MeshEntry&, const Transform& placement)
{
    const double sx{readNumber(line, "a scale factor")};
    const auto next{line.peek()};
    if (!next || startsInstanceWord(*next)) {
        return Transform::scaling({sx, sx, sx}) * placement;
    }
    const double sy{readNumber(line, "the y scale factor")};
    const double sz{readNumber(line, "the z scale factor")};
    return Transform::scaling({sx, sy, sz}) * placement;
}

Transform rotateOperation(SceneState&, LineWords& line, const MeshEntry&, const Transform& placement)
{
    const Vec3 axis{readPoint(line, "the rotation axis")};
    return Transform::rotation(axis, readNumber(line, "the rotation angle")) * placement;
}

// 'fit size': scales the placed mesh's box about its centre so that its
// largest extent is `size`, and moves that centre to the origin.
Transform fitOperation(SceneState& state, LineWords& line, const MeshEntry& mesh, const Transform& placement)
{
    const double size{readScalar(line, Kind::Positive, "the fitted size", 0, 0)};
    const Box3 box{placement.applyBox(state.scene.meshes[mesh.id].bounds)};
    if (!isFinite(box.min) || !isFinite(box.max)) {
        line.fail("the instance is out of range before 'fit'");
    }
    const Vec3 extent{box.extent()};
    const double factor{size / std::max({extent.x, extent.y, extent.z})};
    if (!std::isfinite(factor) || !(factor > 0)) {
        line.fail("the instance is too large or too small to fit");
    }
    const Vec3 middle{box.min.x / 2 + box.max.x / 2, box.min.y / 2 + box.max.y / 2, box.min.z / 2 + box.max.z / 2};
    return Transform::scaling({factor, factor, factor}) * Transform::translation(-middle) * placement;
}

// 'ground': lifts or lowers the placed mesh so that its lowest used vertex
// sits at y = 0; all 'ground' operations of a file examine at most
// kMaxGroundPoints vertices between them.
Transform groundOperation(SceneState& state, LineWords& line, const MeshEntry& mesh, const Transform& placement)
{
    if (mesh.points.size() > state.ground_points_left) {
        line.fail(std::format("'ground' would examine more than {} points in the scene", kMaxGroundPoints));
    }
    state.ground_points_left -= mesh.points.size();
    double lowest{std::numeric_limits<double>::infinity()};
    for (const Vec3& p : mesh.points) {
        const double height{placement.applyPoint(p).y};
        if (!std::isfinite(height)) {
            line.fail("the instance is out of range before 'ground'");
        }
        lowest = std::min(lowest, height);
    }
    return Transform::translation({0, -lowest, 0}) * placement;
}

constexpr std::array<std::pair<std::string_view, Operation>, 5> kOperations{{
    {"translate", &translateOperation},
    {"scale", &scaleOperation},
    {"rotate", &rotateOperation},
    {"fit", &fitOperation},
    {"ground", &groundOperation},
}};

bool startsInstanceWord(std::string_view word)
{
    return word == "material" ||
           std::ranges::find(kOperations, word, &std::pair<std::string_view, Operation>::first) != kOperations.end();
}

void instanceStatement(SceneState& state, LineWords& line)
{
    state.countObject(line);
    const std::string_view mesh_name{readName(line, "a mesh name")};
    const auto mesh{state.meshes.find(mesh_name)};
    if (mesh == state.meshes.end()) {
        line.fail(std::format("mesh {} is not defined", quoted(mesh_name)));
    }
    std::optional<std::uint32_t> material;
    Transform placement{};
    std::size_t operations{0};
    while (const auto word{line.take()}) {
        if (*word == "material") {
            if (material) {
                line.fail("'material' is given twice");
            }
            material = state.materialNamed(line);
            continue;
        }
        if (++operations > kMaxInstanceOperations) {
            line.fail(std::format("more than {} operations", kMaxInstanceOperations));
        }
        const auto found{std::ranges::find(kOperations, *word, &std::pair<std::string_view, Operation>::first)};
        if (found == kOperations.end()) {
            line.fail(std::format("unknown instance operation {}", quoted(*word)));
        }
        try {
            placement = found->second(state, line, mesh->second, placement);
        } catch (const std::invalid_argument& error) {
            line.fail(error.what());
        }
    }
    if (!material) {
        line.fail("missing 'material'");
    }
    try {
        state.scene.addInstance(mesh->second.id, placement, *material);
    } catch (const std::invalid_argument& error) {
        line.fail(error.what());
    }
}

// ------------------------------------------------ the file

using StatementReader = void (*)(SceneState&, LineWords&);

constexpr std::array<std::pair<std::string_view, StatementReader>, 8> kStatements{{
    {"camera", &cameraStatement},
    {"sky", &skyStatement},
    {"material", &materialStatement},
    {"sphere", &sphereStatement},
    {"point_light", &pointLightStatement},
    {"area_light", &areaLightStatement},
    {"mesh", &meshStatement},
    {"instance", &instanceStatement},
}};

HostScene readSceneStream(std::istream& input, const std::filesystem::path& base_directory)
{
    SceneState state;
    state.directory = base_directory;
    forEachLine(
        input, kMaxSceneLine,
        [&](std::string_view text, std::size_t number) {
            LineWords line{text.substr(0, text.find('#')), number};
            const auto keyword{line.take()};
            if (!keyword) {
                return;
            }
            const auto found{
                std::ranges::find(kStatements, *keyword, &std::pair<std::string_view, StatementReader>::first)};
            if (found == kStatements.end()) {
                line.fail(std::format("unknown statement {}", quoted(*keyword)));
            }
            found->second(state, line);
        },
        [](std::size_t number) {
            throw SceneParseError{number, std::format("line longer than {} bytes", kMaxSceneLine)};
        });
    if (!state.scene.has_camera) {
        throw SceneParseError{0, "the scene has no camera"};
    }
    state.scene.finalize();
    return std::move(state.scene);
}

} // namespace

HostScene readSceneText(const std::string& text, const std::filesystem::path& base_directory)
{
    std::istringstream input{text};
    return readSceneStream(input, base_directory);
}

HostScene readSceneFile(const std::filesystem::path& path)
{
    std::error_code error;
    const auto type{std::filesystem::status(path, error).type()};
    if (!error && type != std::filesystem::file_type::not_found && type != std::filesystem::file_type::regular) {
        throw std::runtime_error{std::format("scene file '{}' is not a regular file", path.string())};
    }
    std::ifstream file{path, std::ios::binary};
    if (!file) {
        throw std::runtime_error{std::format("cannot open scene file '{}'", path.string())};
    }
    std::filesystem::path base{path.parent_path()};
    if (base.empty()) {
        base = ".";
    }
    return readSceneStream(file, base);
}

} // namespace albedo_b200
