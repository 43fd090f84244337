// The standard 3DGS .ply layout (reference src/ply.rs:19-181) read into and written from
// device parameter planes.
//
// Layout: binary little-endian float32 vertices with the properties
// `x y z nx ny nz f_dc_0..2 f_rest_0..(3*(K-1)-1) opacity scale_0..2 rot_0..3`, K = (d+1)^2,
// f_rest channel-major (f_rest[c*(K-1) + (k-1)] is coefficient k of channel c); opacity is
// the logit, scales are logs, the rotation is the unnormalised (w, x, y, z). Reading takes
// the property order from the header, so files from other tools load as long as they use
// float properties with these names. The body goes to the device as raw bytes and one
// kernel per direction converts between the file's rows and the parameter planes.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "renderer.cuh"

namespace splat {

// Column of each model scalar in a file row (59 entries in reference record order; -1 for
// coefficients the file does not carry, which read as 0).
struct PlyColumns {
  int col[59];
};

__global__ void ply_rows_to_planes_kernel(const float* __restrict__ rows, int64_t n, int stride, PlyColumns cols,
                                          float4* __restrict__ planes, int64_t cap) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* r = rows + (size_t)i * stride;
  float a[60];
#pragma unroll
  for (int k = 0; k < 59; k++) a[k] = cols.col[k] >= 0 ? r[cols.col[k]] : 0.0f;
  a[59] = 0.0f;
  planes[i] = make_float4(a[0], a[1], a[2], a[10]);
  planes[cap + i] = make_float4(a[6], a[7], a[8], a[9]);
  planes[2 * cap + i] = make_float4(a[3], a[4], a[5], 0.0f);
#pragma unroll
  for (int q = 0; q < 12; q++) planes[(3 + q) * cap + i] = make_float4(a[11 + 4 * q], a[12 + 4 * q], a[13 + 4 * q], a[14 + 4 * q]);
}

__global__ void ply_planes_to_rows_kernel(const float4* __restrict__ planes, int64_t n, int64_t cap, PlyColumns cols,
                                          int stride, float* __restrict__ rows) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float a[60];
  const float4 p0 = planes[i], p1 = planes[cap + i], p2 = planes[2 * cap + i];
  a[0] = p0.x;
  a[1] = p0.y;
  a[2] = p0.z;
  a[10] = p0.w;
  a[6] = p1.x;
  a[7] = p1.y;
  a[8] = p1.z;
  a[9] = p1.w;
  a[3] = p2.x;
  a[4] = p2.y;
  a[5] = p2.z;
#pragma unroll
  for (int q = 0; q < 12; q++) {
    const float4 s = planes[(3 + q) * cap + i];
    a[11 + 4 * q] = s.x;
    a[12 + 4 * q] = s.y;
    a[13 + 4 * q] = s.z;
    a[14 + 4 * q] = s.w;
  }
  float* r = rows + (size_t)i * stride;
  for (int c = 0; c < stride; c++) r[c] = 0.0f;  // normals and absent columns
#pragma unroll
  for (int k = 0; k < 59; k++)
    if (cols.col[k] >= 0) r[cols.col[k]] = a[k];
}

namespace {

int num_coeffs(int degree) { return (degree + 1) * (degree + 1); }

// Columns of the layout this library writes for a degree (ply.rs:19-69).
void write_columns(int degree, PlyColumns* cols, int* stride, std::string* header_props) {
  const int K = num_coeffs(degree);
  const int n_rest = 3 * (K - 1);
  for (int k = 0; k < 59; k++) cols->col[k] = -1;
  std::string h;
  const char* first[] = {"x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"};
  for (const char* nm : first) h += std::string("property float ") + nm + "\n";
  for (int i = 0; i < n_rest; i++) h += "property float f_rest_" + std::to_string(i) + "\n";
  h += "property float opacity\n";
  for (int i = 0; i < 3; i++) h += "property float scale_" + std::to_string(i) + "\n";
  for (int i = 0; i < 4; i++) h += "property float rot_" + std::to_string(i) + "\n";
  // record index -> column
  for (int i = 0; i < 3; i++) cols->col[i] = i;                  // mean
  for (int c = 0; c < 3; c++) cols->col[11 + c] = 6 + c;          // sh[0][c]
  for (int c = 0; c < 3; c++)
    for (int k = 1; k < K; k++) cols->col[11 + 3 * k + c] = 9 + c * (K - 1) + (k - 1);
  cols->col[10] = 9 + n_rest;                                     // opacity
  for (int i = 0; i < 3; i++) cols->col[3 + i] = 10 + n_rest + i; // log_scale
  for (int i = 0; i < 4; i++) cols->col[6 + i] = 13 + n_rest + i; // quat
  *stride = 17 + n_rest;
  *header_props = h;
}

Status fmt_error(const std::string& path, const std::string& m) {
  return Status::make(SPLAT_ERR_INVALID, path + ": " + m);
}

// Parses the header (ply.rs:76-151). On success fills the columns, the vertex count, the
// row stride in floats, the degree and the byte offset of the body.
// `bytes` holds at least the header; `file_size` is the size of the whole file.
Status parse_header(const std::string& path, const std::vector<char>& bytes, size_t file_size, PlyColumns* cols,
                    int64_t* count, int* stride, int* degree, size_t* body) {
  const char* needle = "end_header\n";
  const size_t nl = strlen(needle);
  size_t end = std::string::npos;
  for (size_t i = 0; i + nl <= bytes.size(); i++)
    if (memcmp(&bytes[i], needle, nl) == 0) {
      end = i;
      break;
    }
  if (end == std::string::npos) return fmt_error(path, "missing end_header");
  std::string header(bytes.data(), end);
  std::vector<std::string> props;
  bool in_vertex = false, binary_le = false, have_count = false;
  int64_t n = 0;
  size_t pos = 0;
  while (pos < header.size()) {
    size_t e = header.find('\n', pos);
    if (e == std::string::npos) e = header.size();
    std::string line = header.substr(pos, e - pos);
    pos = e + 1;
    std::vector<std::string> t;
    size_t p = 0;
    while (p < line.size()) {
      while (p < line.size() && isspace((unsigned char)line[p])) p++;
      size_t q = p;
      while (q < line.size() && !isspace((unsigned char)line[q])) q++;
      if (q > p) t.push_back(line.substr(p, q - p));
      p = q;
    }
    if (t.empty()) continue;
    if (t[0] == "format") {
      if (t.size() == 3 && t[1] == "binary_little_endian")
        binary_le = true;
      else
        return fmt_error(path, "only binary_little_endian is supported");
    } else if (t[0] == "element") {
      if (t.size() == 3 && t[1] == "vertex") {
        in_vertex = true;
        char* endp = nullptr;
        const long long v = strtoll(t[2].c_str(), &endp, 10);
        if (!endp || *endp != 0 || v < 0) return fmt_error(path, "bad vertex count");
        n = v;
        have_count = true;
      } else {
        in_vertex = false;
      }
    } else if (t[0] == "property" && t.size() == 3 && in_vertex) {
      if (t[1] != "float" && t[1] != "float32")
        return fmt_error(path, "property " + t[2] + " has type " + t[1] + "; only float is supported");
      props.push_back(t[2]);
    }
  }
  if (!binary_le) return fmt_error(path, "missing format line");
  if (!have_count) return fmt_error(path, "missing vertex element");
  const int64_t st = (int64_t)props.size();
  const size_t body_off = end + nl;
  if (st > 0 && n > (int64_t)((file_size - body_off) / (size_t)(st * 4)))
    return fmt_error(path, "file is shorter than the header announces");
  auto index = [&](const std::string& name, int* out) -> Status {
    for (size_t i = 0; i < props.size(); i++)
      if (props[i] == name) {
        *out = (int)i;
        return Status::ok();
      }
    return fmt_error(path, "missing property " + name);
  };
  for (int k = 0; k < 59; k++) cols->col[k] = -1;
  const char* xyz[] = {"x", "y", "z"};
  for (int i = 0; i < 3; i++) SPLAT_TRY(index(xyz[i], &cols->col[i]));
  for (int i = 0; i < 3; i++) SPLAT_TRY(index("f_dc_" + std::to_string(i), &cols->col[11 + i]));
  SPLAT_TRY(index("opacity", &cols->col[10]));
  for (int i = 0; i < 3; i++) SPLAT_TRY(index("scale_" + std::to_string(i), &cols->col[3 + i]));
  for (int i = 0; i < 4; i++) SPLAT_TRY(index("rot_" + std::to_string(i), &cols->col[6 + i]));
  int n_rest = 0;
  for (const auto& pnm : props)
    if (pnm.rfind("f_rest_", 0) == 0) n_rest++;
  int d;
  switch (n_rest) {
    case 0: d = 0; break;
    case 9: d = 1; break;
    case 24: d = 2; break;
    case 45: d = 3; break;
    default: return fmt_error(path, "unsupported number of f_rest properties: " + std::to_string(n_rest));
  }
  const int K = num_coeffs(d);
  for (int c = 0; c < 3; c++)
    for (int k = 1; k < K; k++) SPLAT_TRY(index("f_rest_" + std::to_string(c * (K - 1) + (k - 1)), &cols->col[11 + 3 * k + c]));
  *count = n;
  *stride = (int)st;
  *degree = d;
  *body = body_off;
  return Status::ok();
}

}  // namespace

}  // namespace splat

using namespace splat;

extern "C" {

SPLAT_API int splat_ply_read_header(splat_ctx* ctx, const char* path, int64_t* count, int32_t* sh_degree) {
  if (!ctx) return SPLAT_ERR_INVALID;
  Ctx* c = splat_ctx_impl(ctx);
  if (!path || !count || !sh_degree) {
    c->last_error = "splat_ply_read_header: bad arguments";
    return SPLAT_ERR_INVALID;
  }
  FILE* f = fopen(path, "rb");
  if (!f) {
    c->last_error = std::string(path) + ": cannot open";
    return SPLAT_ERR_INVALID;
  }
  std::vector<char> head(1 << 16);
  const size_t got = fread(head.data(), 1, head.size(), f);
  fseek(f, 0, SEEK_END);
  const long size = ftell(f);
  fclose(f);
  head.resize(got);
  PlyColumns cols;
  int64_t n = 0;
  int stride = 0, degree = 0;
  size_t body = 0;
  Status s = parse_header(path, head, size > 0 ? (size_t)size : 0, &cols, &n, &stride, &degree, &body);
  if (!s.good()) {
    c->last_error = s.msg;
    return s.code;
  }
  *count = n;
  *sh_degree = degree;
  return SPLAT_OK;
}

// read (ply.rs:73-181) into parameter planes of capacity cap >= count.
SPLAT_API int splat_ply_read(splat_ctx* ctx, const char* path, float* planes_dev, int64_t cap, int64_t* count,
                             int32_t* sh_degree) {
  if (!ctx) return SPLAT_ERR_INVALID;
  Ctx* c = splat_ctx_impl(ctx);
  if (!path || !planes_dev || !count || !sh_degree) {
    c->last_error = "splat_ply_read: bad arguments";
    return SPLAT_ERR_INVALID;
  }
  FILE* f = fopen(path, "rb");
  if (!f) {
    c->last_error = std::string(path) + ": cannot open";
    return SPLAT_ERR_INVALID;
  }
  fseek(f, 0, SEEK_END);
  const long size = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<char> bytes(size > 0 ? (size_t)size : 0);
  const size_t got = size > 0 ? fread(bytes.data(), 1, bytes.size(), f) : 0;
  fclose(f);
  if (got != bytes.size()) {
    c->last_error = std::string(path) + ": short read";
    return SPLAT_ERR_INVALID;
  }
  PlyColumns cols;
  int64_t n = 0;
  int stride = 0, degree = 0;
  size_t body = 0;
  Status s = parse_header(path, bytes, bytes.size(), &cols, &n, &stride, &degree, &body);
  if (s.good() && n > cap) s = Status::make(SPLAT_ERR_CAPACITY, "splat_ply_read: the file holds more Gaussians than cap");
  if (!s.good()) {
    c->last_error = s.msg;
    return s.code;
  }
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != c->device) cudaSetDevice(c->device);
  arena_reset(c);
  float* rows = nullptr;
  const size_t nbytes = (size_t)n * stride * 4;
  if (n > 0) {
    s = arena_reserve(c, nbytes, (void**)&rows);
    if (s.good()) s = cuda_status(cudaMemcpyAsync(rows, bytes.data() + body, nbytes, cudaMemcpyHostToDevice, c->stream),
                                  "upload ply body");
    if (s.good()) {
      ply_rows_to_planes_kernel<<<ceil_div(n, 256), 256, 0, c->stream>>>(rows, n, stride, cols,
                                                                         reinterpret_cast<float4*>(planes_dev), cap);
      c->launches.count++;
      s = cuda_status(cudaGetLastError(), "ply_rows_to_planes_kernel");
    }
    if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  }
  if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
  if (!s.good()) {
    c->last_error = s.msg;
    return s.code;
  }
  *count = n;
  *sh_degree = degree;
  return SPLAT_OK;
}

// write (ply.rs:19-69) from parameter planes; coefficients above sh_degree are not written.
SPLAT_API int splat_ply_write(splat_ctx* ctx, const char* path, const float* planes_dev, int64_t n, int64_t cap,
                              int32_t sh_degree) {
  if (!ctx) return SPLAT_ERR_INVALID;
  Ctx* c = splat_ctx_impl(ctx);
  if (!path || n < 0 || cap < n || (n && !planes_dev) || sh_degree < 0 || sh_degree > 3) {
    c->last_error = "splat_ply_write: bad arguments";
    return SPLAT_ERR_INVALID;
  }
  PlyColumns cols;
  int stride = 0;
  std::string props;
  write_columns(sh_degree, &cols, &stride, &props);
  std::string header = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(n) + "\n" + props +
                       "end_header\n";
  std::vector<char> body((size_t)n * stride * 4);
  Status s = Status::ok();
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != c->device) cudaSetDevice(c->device);
  arena_reset(c);
  if (n > 0) {
    float* rows = nullptr;
    s = arena_reserve(c, body.size(), (void**)&rows);
    if (s.good()) {
      ply_planes_to_rows_kernel<<<ceil_div(n, 256), 256, 0, c->stream>>>(reinterpret_cast<const float4*>(planes_dev),
                                                                         n, cap, cols, stride, rows);
      c->launches.count++;
      s = cuda_status(cudaGetLastError(), "ply_planes_to_rows_kernel");
    }
    if (s.good())
      s = cuda_status(cudaMemcpyAsync(body.data(), rows, body.size(), cudaMemcpyDeviceToHost, c->stream),
                      "download rows");
    if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  }
  if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
  if (!s.good()) {
    c->last_error = s.msg;
    return s.code;
  }
  FILE* f = fopen(path, "wb");
  if (!f) {
    c->last_error = std::string(path) + ": cannot create";
    return SPLAT_ERR_INVALID;
  }
  bool ok = fwrite(header.data(), 1, header.size(), f) == header.size();
  if (ok && !body.empty()) ok = fwrite(body.data(), 1, body.size(), f) == body.size();
  ok = (fclose(f) == 0) && ok;
  if (!ok) {
    c->last_error = std::string(path) + ": write failed";
    return SPLAT_ERR_INVALID;
  }
  return SPLAT_OK;
}

}  // extern "C"
