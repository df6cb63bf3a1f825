// Scene-file and OBJ reading. Restates scene/scene_file.cpp (grammar, value
// ranges, limits, mesh path rules, instance operations) and geometry/obj.cpp
// (v / vt / f statements, fan triangulation, negative indices), with numbers
// parsed by std::from_chars exactly as io/tokens.cpp:25-52 parses them.
#include "scene_file.hpp"

#include <algorithm>
#include <charconv>
#include <format>
#include <fstream>
#include <functional>
#include <map>
#include <optional>
#include <sstream>
#include <string_view>
#include <thread>
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
        std::vector<std::thread> workers;
        for (std::size_t k{1}; k < parts.size(); ++k) {
            workers.emplace_back([&, k] { work(k); });
        }
        if (!parts.empty()) {
            work(0);
        }
        for (std::thread& worker : workers) {
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

class Statement {
public:
    Statement(std::string_view text, std::size_t line) : words{text}, line_number{line} {}

    [[noreturn]] void fail(const std::string& problem) const { throw SceneParseError{line_number, problem}; }
    std::optional<std::string_view> next() { return words.next(); }
    std::optional<std::string_view> peek() const
    {
        Words rest{words};
        return rest.next();
    }
    std::string_view word(std::string_view what)
    {
        const auto token{next()};
        if (!token) {
            fail(std::format("expected {}", what));
        }
        return *token;
    }
    double number(std::string_view what)
    {
        const std::string_view token{word(what)};
        const auto value{parseReal(token)};
        if (!value) {
            fail(std::format("{} must be a finite number, got {}", what, quoted(token)));
        }
        return *value;
    }
    double inRange(std::string_view what, double low, double high)
    {
        const double value{number(what)};
        if (value < low || value > high) {
            fail(std::format("{} must be between {} and {}, got {}", what, low, high, value));
        }
        return value;
    }
    double positive(std::string_view what)
    {
        const double value{number(what)};
        if (!(value > 0)) {
            fail(std::format("{} must be positive, got {}", what, value));
        }
        return value;
    }
    Vec3 point(std::string_view what)
    {
        const double x{number(std::format("the x coordinate of {}", what))};
        const double y{number(std::format("the y coordinate of {}", what))};
        return {x, y, number(std::format("the z coordinate of {}", what))};
    }
    Rgb color(std::string_view what, double low, double high)
    {
        const double r{inRange(std::format("the red channel of {}", what), low, high)};
        const double g{inRange(std::format("the green channel of {}", what), low, high)};
        return {r, g, inRange(std::format("the blue channel of {}", what), low, high)};
    }
    Rgb reflectance(std::string_view what) { return color(what, 0, kMaxReflectance); }
    Rgb emission(std::string_view what) { return color(what, 0, kMaxEmission); }
    std::string_view name(std::string_view what)
    {
        const std::string_view token{word(what)};
        if (!isIdentifier(token)) {
            fail(std::format("{} is not a valid name", quoted(token)));
        }
        return token;
    }
    template <typename Read>
    void readFields(Read read)
    {
        std::vector<std::string_view> seen;
        while (const auto field{next()}) {
            if (std::ranges::find(seen, *field) != seen.end()) {
                fail(std::format("{} is given twice", quoted(*field)));
            }
            seen.push_back(*field);
            if (!read(*field)) {
                fail(std::format("unknown field {}", quoted(*field)));
            }
        }
    }
    template <typename T>
    T required(const std::optional<T>& value, std::string_view what) const
    {
        if (!value) {
            fail(std::format("missing '{}'", what));
        }
        return *value;
    }
    void expectEnd()
    {
        if (const auto extra{next()}) {
            fail(std::format("unexpected {}", quoted(*extra)));
        }
    }

private:
    Words words;
    std::size_t line_number;
};

struct LoadedMesh {
    std::uint32_t id{};
    std::vector<Vec3> points; // positions used by kept triangles, each once
};

bool isInstanceKeyword(std::string_view word)
{
    constexpr std::array<std::string_view, 6> keywords{"material", "translate", "scale", "rotate", "fit", "ground"};
    return std::ranges::find(keywords, word) != keywords.end();
}

// A relative path without '..', control bytes or a root (scene/scene_file.cpp:368-395),
// resolved inside `base` (scene/scene_file.cpp:400-430).
std::filesystem::path meshFile(const Statement& statement, const std::filesystem::path& base, std::string_view text)
{
    const bool control{std::ranges::any_of(text, [](char c) {
        const auto byte{static_cast<unsigned char>(c)};
        return byte < 0x20 || byte == 0x7F;
    })};
    if (control) {
        statement.fail(std::format("mesh path {} must be UTF-8 without control characters", quoted(text)));
    }
    const std::filesystem::path relative{std::string{text}};
    if (relative.is_absolute() || relative.has_root_name() || relative.has_root_directory() ||
        std::ranges::find(relative, std::filesystem::path{".."}) != relative.end()) {
        statement.fail(std::format("mesh path {} must be relative to the scene and not use '..'", quoted(text)));
    }
    std::error_code error;
    const std::filesystem::path real_base{std::filesystem::canonical(base, error)};
    if (error) {
        statement.fail("the scene's directory cannot be resolved");
    }
    const std::filesystem::path real_file{std::filesystem::weakly_canonical(real_base / relative, error)};
    if (error) {
        statement.fail(std::format("cannot resolve mesh path {}", quoted(text)));
    }
    const auto [base_end, file_part]{std::ranges::mismatch(real_base, real_file)};
    if (base_end != real_base.end()) {
        statement.fail(std::format("mesh path {} leads outside the scene's directory", quoted(text)));
    }
    const auto status{std::filesystem::status(real_file, error)};
    if (status.type() == std::filesystem::file_type::not_found) {
        statement.fail(std::format("mesh file {} does not exist", quoted(text)));
    }
    if (status.type() != std::filesystem::file_type::regular) {
        statement.fail(std::format("mesh path {} is not a regular file", quoted(text)));
    }
    return real_file;
}

class SceneReader {
public:
    explicit SceneReader(std::filesystem::path directory) : base_directory{std::move(directory)} {}

    void readLine(std::string_view line, std::size_t line_number)
    {
        Statement statement{line.substr(0, line.find('#')), line_number};
        const auto keyword{statement.next()};
        if (!keyword) {
            return;
        }
        if (*keyword == "camera") {
            readCamera(statement);
        } else if (*keyword == "sky") {
            readSky(statement);
        } else if (*keyword == "material") {
            readMaterial(statement);
        } else if (*keyword == "sphere") {
            readSphere(statement);
        } else if (*keyword == "point_light") {
            readPointLight(statement);
        } else if (*keyword == "area_light") {
            readAreaLight(statement);
        } else if (*keyword == "mesh") {
            readMesh(statement);
        } else if (*keyword == "instance") {
            readInstance(statement);
        } else {
            statement.fail(std::format("unknown statement {}", quoted(*keyword)));
        }
    }

    HostScene finish() &&
    {
        if (!scene.has_camera) {
            throw SceneParseError{0, "the scene has no camera"};
        }
        scene.finalize();
        return std::move(scene);
    }

private:
    void readCamera(Statement& statement)
    {
        if (scene.has_camera) {
            statement.fail("the scene already has a camera");
        }
        std::optional<Vec3> from;
        std::optional<Vec3> at;
        CameraSettings settings{};
        statement.readFields([&](std::string_view field) {
            if (field == "from") {
                from = statement.point("the camera position");
            } else if (field == "at") {
                at = statement.point("the point the camera looks at");
            } else if (field == "up") {
                settings.up = statement.point("the camera's up direction");
            } else if (field == "fov") {
                settings.vertical_fov_degrees = statement.number("the field of view");
            } else {
                return false;
            }
            return true;
        });
        settings.look_from = statement.required(from, "from");
        settings.look_at = statement.required(at, "at");
        try {
            static_cast<void>(buildCameraFrame(settings, 16.0 / 9.0));
        } catch (const std::invalid_argument& error) {
            statement.fail(error.what());
        }
        scene.camera = settings;
        scene.has_camera = true;
    }

    void readSky(Statement& statement)
    {
        if (sky_given) {
            statement.fail("the scene already has a sky");
        }
        const auto first{statement.peek()};
        if (first && (*first == "nadir" || *first == "zenith")) {
            std::optional<Rgb> nadir;
            std::optional<Rgb> zenith;
            statement.readFields([&](std::string_view field) {
                if (field == "nadir") {
                    nadir = statement.emission("the radiance from below");
                } else if (field == "zenith") {
                    zenith = statement.emission("the radiance from above");
                } else {
                    return false;
                }
                return true;
            });
            scene.setSky(statement.required(nadir, "nadir"), statement.required(zenith, "zenith"));
        } else {
            const Rgb radiance{statement.emission("the sky's radiance")};
            statement.expectEnd();
            scene.setSky(radiance, radiance);
        }
        sky_given = true;
    }

    void readMaterial(Statement& statement)
    {
        if (material_ids.size() >= kMaxMaterials) {
            statement.fail(std::format("more than {} materials", kMaxMaterials));
        }
        const std::string_view name{statement.name("a material name")};
        if (material_ids.contains(name)) {
            statement.fail(std::format("material {} is already defined", quoted(name)));
        }
        const std::string_view type{statement.word("a material type")};
        MaterialDesc material;
        if (type == "mix") {
            material = readMix(statement);
        } else {
            material.first = basicOfType(statement, type);
        }
        material_ids.emplace(std::string{name}, scene.addMaterial(material));
    }

    static BasicMaterialDesc basicOfType(Statement& statement, std::string_view type)
    {
        BasicMaterialDesc basic;
        if (type == "diffuse") {
            std::optional<Rgb> color;
            statement.readFields([&](std::string_view field) {
                if (field != "color") {
                    return false;
                }
                color = statement.reflectance("the color");
                return true;
            });
            basic.texture = {TextureKind::Constant, statement.required(color, "color")};
        } else if (type == "checker") {
            std::optional<Rgb> even;
            std::optional<Rgb> odd;
            std::optional<double> frequency;
            statement.readFields([&](std::string_view field) {
                if (field == "even") {
                    even = statement.reflectance("the even color");
                } else if (field == "odd") {
                    odd = statement.reflectance("the odd color");
                } else if (field == "frequency") {
                    frequency = statement.positive("the checker frequency");
                } else {
                    return false;
                }
                return true;
            });
            basic.texture = {TextureKind::Checker, statement.required(even, "even"), statement.required(odd, "odd"),
                             statement.required(frequency, "frequency")};
        } else if (type == "perlin") {
            std::optional<Rgb> low;
            std::optional<Rgb> high;
            std::optional<double> scale;
            double veins{0};
            statement.readFields([&](std::string_view field) {
                if (field == "low") {
                    low = statement.reflectance("the low color");
                } else if (field == "high") {
                    high = statement.reflectance("the high color");
                } else if (field == "scale") {
                    scale = statement.positive("the noise scale");
                } else if (field == "veins") {
                    veins = statement.inRange("the veins", 0, kMaxPerlinVeins);
                } else {
                    return false;
                }
                return true;
            });
            basic.texture = {TextureKind::Perlin, statement.required(low, "low"), statement.required(high, "high"),
                             statement.required(scale, "scale"), veins};
        } else if (type == "conductor") {
            std::optional<Rgb> eta;
            std::optional<Rgb> k;
            double roughness{0};
            statement.readFields([&](std::string_view field) {
                if (field == "eta") {
                    eta = statement.color("the refractive index", kMinConductorEta, kMaxConductorEta);
                } else if (field == "k") {
                    k = statement.color("the absorption", 0, kMaxConductorK);
                } else if (field == "roughness") {
                    roughness = statement.inRange("the roughness", 0, kMaxRoughness);
                } else {
                    return false;
                }
                return true;
            });
            basic.kind = BasicKind::Conductor;
            basic.eta = statement.required(eta, "eta");
            basic.k = statement.required(k, "k");
            basic.roughness = roughness;
            const std::array<double, 3> e{basic.eta.r, basic.eta.g, basic.eta.b};
            const std::array<double, 3> a{basic.k.r, basic.k.g, basic.k.b};
            for (std::size_t c{0}; c < 3; ++c) {
                if (e[c] == 1 && a[c] == 0) {
                    statement.fail("a conductor channel cannot have eta 1 and k 0");
                }
            }
        } else if (type == "dielectric") {
            std::optional<double> ior;
            double roughness{0};
            statement.readFields([&](std::string_view field) {
                if (field == "ior") {
                    ior = statement.inRange("the index of refraction", kMinIor, kMaxIor);
                } else if (field == "roughness") {
                    roughness = statement.inRange("the roughness", 0, kMaxRoughness);
                } else {
                    return false;
                }
                return true;
            });
            basic.kind = BasicKind::Dielectric;
            basic.ior = statement.required(ior, "ior");
            basic.roughness = roughness;
        } else {
            statement.fail(std::format("unknown material type {}", quoted(type)));
        }
        return basic;
    }

    MaterialDesc readMix(Statement& statement) const
    {
        std::optional<BasicMaterialDesc> first;
        std::optional<BasicMaterialDesc> second;
        std::optional<double> scale;
        double veins{0};
        double threshold{0.5};
        statement.readFields([&](std::string_view field) {
            if (field == "first") {
                first = basicNamed(statement);
            } else if (field == "second") {
                second = basicNamed(statement);
            } else if (field == "scale") {
                scale = statement.positive("the noise scale");
            } else if (field == "veins") {
                veins = statement.inRange("the veins", 0, kMaxPerlinVeins);
            } else if (field == "threshold") {
                threshold = statement.inRange("the threshold", 0, 1);
            } else {
                return false;
            }
            return true;
        });
        MaterialDesc mix;
        mix.mix = true;
        mix.first = statement.required(first, "first");
        mix.second = statement.required(second, "second");
        mix.scale = statement.required(scale, "scale");
        mix.veins = veins;
        mix.threshold = threshold;
        return mix;
    }

    BasicMaterialDesc basicNamed(Statement& statement) const
    {
        const std::string_view name{statement.peek().value_or("")};
        const MaterialDesc& material{scene.materials[materialNamed(statement)]};
        if (material.mix) {
            statement.fail(std::format("material {} is a mix, and a mix cannot hold another mix", quoted(name)));
        }
        return material.first;
    }

    std::uint32_t materialNamed(Statement& statement) const
    {
        const std::string_view name{statement.name("a material name")};
        const auto found{material_ids.find(name)};
        if (found == material_ids.end()) {
            statement.fail(std::format("material {} is not defined", quoted(name)));
        }
        return found->second;
    }

    void countObject(const Statement& statement)
    {
        if (object_count >= kMaxObjects) {
            statement.fail(std::format("more than {} objects", kMaxObjects));
        }
        ++object_count;
    }

    void readSphere(Statement& statement)
    {
        countObject(statement);
        const Vec3 center{statement.point("the sphere center")};
        std::optional<double> radius;
        std::optional<std::uint32_t> material;
        statement.readFields([&](std::string_view field) {
            if (field == "radius") {
                radius = statement.number("a radius");
            } else if (field == "material") {
                material = materialNamed(statement);
            } else {
                return false;
            }
            return true;
        });
        const double r{statement.required(radius, "radius")};
        try {
            validateSphere(center, r);
        } catch (const std::invalid_argument& error) {
            statement.fail(error.what());
        }
        if (!material) {
            statement.fail("missing 'material'");
        }
        scene.addSphere(center, r, *material);
    }

    void readPointLight(Statement& statement)
    {
        countObject(statement);
        const Vec3 position{statement.point("the light position")};
        std::optional<Rgb> intensity;
        statement.readFields([&](std::string_view field) {
            if (field != "intensity") {
                return false;
            }
            intensity = statement.emission("the intensity");
            return true;
        });
        scene.addPointLight(position, statement.required(intensity, "intensity"));
    }

    void readAreaLight(Statement& statement)
    {
        countObject(statement);
        const Vec3 center{statement.point("the light center")};
        std::optional<double> radius;
        std::optional<Rgb> radiance;
        std::optional<std::uint32_t> material;
        statement.readFields([&](std::string_view field) {
            if (field == "radius") {
                radius = statement.number("a radius");
            } else if (field == "radiance") {
                radiance = statement.emission("the radiance");
            } else if (field == "material") {
                material = materialNamed(statement);
            } else {
                return false;
            }
            return true;
        });
        const double r{statement.required(radius, "radius")};
        try {
            validateSphere(center, r);
        } catch (const std::invalid_argument& error) {
            statement.fail(error.what());
        }
        const Rgb emitted{statement.required(radiance, "radiance")};
        if (!material) {
            // An area light without a material is black diffuse (scene/scene_file.cpp:819).
            material = scene.addMaterial(MaterialDesc{});
        }
        scene.addAreaLight(center, r, emitted, *material);
    }

    void readMesh(Statement& statement)
    {
        if (base_directory.empty()) {
            statement.fail("meshes can only be read from a scene file, which they sit beside");
        }
        if (meshes.size() >= kMaxMeshes) {
            statement.fail(std::format("more than {} meshes", kMaxMeshes));
        }
        const std::string_view name{statement.name("a mesh name")};
        if (meshes.contains(name)) {
            statement.fail(std::format("mesh {} is already defined", quoted(name)));
        }
        const std::string_view path{statement.word("a mesh file")};
        const bool smooth{statement.peek() == "smooth"};
        if (smooth) {
            static_cast<void>(statement.next());
        }
        statement.expectEnd();
        const std::filesystem::path file{meshFile(statement, base_directory, path)};
        ObjMesh obj;
        try {
            obj = readObj(file, budget);
        } catch (const ObjError& error) {
            statement.fail(std::format("mesh {}: {}", quoted(path), error.what()));
        } catch (const std::runtime_error&) {
            statement.fail(std::format("cannot read mesh file {}", quoted(path)));
        }
        LoadedMesh loaded;
        std::vector<bool> used(obj.positions.size(), false);
        for (const auto& f : obj.faces) {
            if (formsTriangle(obj.positions[f[0]], obj.positions[f[1]], obj.positions[f[2]])) {
                used[f[0]] = used[f[1]] = used[f[2]] = true;
            }
        }
        for (std::size_t i{0}; i < obj.positions.size(); ++i) {
            if (used[i]) {
                loaded.points.push_back(obj.positions[i]);
            }
        }
        if (loaded.points.empty()) {
            statement.fail(std::format("mesh {} has no triangles", quoted(path)));
        }
        try {
            loaded.id = scene.addMesh(obj.positions, obj.faces, obj.uvs, obj.texture_faces, smooth);
        } catch (const std::exception& error) {
            statement.fail(std::format("mesh {}: {}", quoted(path), error.what()));
        }
        budget.vertices -= obj.positions.size();
        budget.texture_coordinates -= obj.uvs.size();
        budget.triangles -= obj.faces.size();
        meshes.emplace(std::string{name}, std::move(loaded));
    }

    void readInstance(Statement& statement)
    {
        countObject(statement);
        const std::string_view mesh_name{statement.name("a mesh name")};
        const auto found{meshes.find(mesh_name)};
        if (found == meshes.end()) {
            statement.fail(std::format("mesh {} is not defined", quoted(mesh_name)));
        }
        const LoadedMesh& mesh{found->second};
        std::optional<std::uint32_t> material;
        Transform placement{};
        std::size_t operations{0};
        while (const auto word{statement.next()}) {
            if (*word == "material") {
                if (material) {
                    statement.fail("'material' is given twice");
                }
                material = materialNamed(statement);
                continue;
            }
            if (++operations > kMaxInstanceOperations) {
                statement.fail(std::format("more than {} operations", kMaxInstanceOperations));
            }
            placement = applied(statement, *word, mesh, placement);
        }
        if (!material) {
            statement.fail("missing 'material'");
        }
        try {
            scene.addInstance(mesh.id, placement, *material);
        } catch (const std::invalid_argument& error) {
            statement.fail(error.what());
        }
    }

    // scene/scene_file.cpp:962-1038.
    Transform applied(Statement& statement, std::string_view name, const LoadedMesh& mesh, const Transform& placement)
    {
        try {
            if (name == "translate") {
                return Transform::translation(statement.point("the translation")) * placement;
            }
            if (name == "scale") {
                const double first{statement.number("a scale factor")};
                const auto next{statement.peek()};
                if (!next || isInstanceKeyword(*next)) {
                    return Transform::scaling({first, first, first}) * placement;
                }
                const double y{statement.number("the y scale factor")};
                return Transform::scaling({first, y, statement.number("the z scale factor")}) * placement;
            }
            if (name == "rotate") {
                const Vec3 axis{statement.point("the rotation axis")};
                return Transform::rotation(axis, statement.number("the rotation angle")) * placement;
            }
            if (name == "fit") {
                const double size{statement.positive("the fitted size")};
                const Box3 box{placement.applyBox(scene.meshes[mesh.id].bounds)};
                if (!isFinite(box.min) || !isFinite(box.max)) {
                    statement.fail("the instance is out of range before 'fit'");
                }
                const Vec3 extent{box.extent()};
                const double scale{size / std::max({extent.x, extent.y, extent.z})};
                if (!std::isfinite(scale) || !(scale > 0)) {
                    statement.fail("the instance is too large or too small to fit");
                }
                const Vec3 center{box.min.x / 2 + box.max.x / 2, box.min.y / 2 + box.max.y / 2,
                                  box.min.z / 2 + box.max.z / 2};
                return Transform::scaling({scale, scale, scale}) * Transform::translation(-center) * placement;
            }
            if (name == "ground") {
                if (mesh.points.size() > ground_points_left) {
                    statement.fail(
                        std::format("'ground' would examine more than {} points in the scene", kMaxGroundPoints));
                }
                ground_points_left -= mesh.points.size();
                std::optional<double> lowest;
                for (const Vec3& p : mesh.points) {
                    const double height{placement.applyPoint(p).y};
                    if (!std::isfinite(height)) {
                        lowest.reset();
                        break;
                    }
                    lowest = lowest ? std::min(*lowest, height) : height;
                }
                if (!lowest) {
                    statement.fail("the instance is out of range before 'ground'");
                }
                return Transform::translation({0, -*lowest, 0}) * placement;
            }
        } catch (const std::invalid_argument& error) {
            statement.fail(error.what());
        }
        statement.fail(std::format("unknown instance operation {}", quoted(name)));
    }

    std::filesystem::path base_directory;
    HostScene scene;
    bool sky_given{false};
    std::map<std::string, std::uint32_t, std::less<>> material_ids;
    std::map<std::string, LoadedMesh, std::less<>> meshes;
    ObjBudget budget{};
    std::size_t ground_points_left{kMaxGroundPoints};
    std::size_t object_count{0};
};

HostScene readSceneStream(std::istream& input, const std::filesystem::path& base_directory)
{
    SceneReader reader{base_directory};
    forEachLine(
        input, kMaxSceneLine, [&](std::string_view line, std::size_t number) { reader.readLine(line, number); },
        [](std::size_t number) { throw SceneParseError{number, std::format("line longer than {} bytes", kMaxSceneLine)}; });
    return std::move(reader).finish();
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
