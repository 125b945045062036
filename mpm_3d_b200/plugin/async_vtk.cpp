// AsyncVTK: DefaultVTK's frames written by a background thread (see
// async_vtk.hpp).
#include "async_vtk.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "job.hpp"
#include "mpm_tensorarray.hpp"
#include "mpm_vectorarray.hpp"
#include "parser.hpp"

AsyncVTK::AsyncVTK() {
  object_name = "AsyncVTK";
  mainpath = "";
  // the streams the objects write into keep their text in memory
  static_cast<std::ios&>(pcap_).rdbuf(&pbuf_);
  static_cast<std::ios&>(ncap_).rdbuf(&nbuf_);
}

AsyncVTK::~AsyncVTK() {
  {
    std::lock_guard<std::mutex> lock(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  if (writer_.joinable()) writer_.join();
}

// DefaultVTK::init (default_vtk.cpp:25-50): the same properties, the same
// exit(0) on missing ones; int-properties[0] sets maxPending.
void AsyncVTK::init(Job* job) {
  if (str_props.size() < 3 || fp64_props.size() < 1) {
    std::cout << str_props.size() << "\n";
    fprintf(stderr, "%s:%s: Need at least 4 properties defined ({sampleRate}, {frameDirectory, outputDirectory, outputName}).\n",
            __FILE__, __func__);
    exit(0);
  }
  frameDirectory = Parser::makeDirectory(str_props[0]);
  outputDirectory = Parser::makeDirectory(str_props[1]);
  outputName = str_props[2];
  sampleRate = fp64_props[0];
  sampledFrames = 0;
  if (!int_props.empty() && int_props[0] > 0) maxPending = int_props[0];
  printf("Serializer properties (frameDirectory = %s, outputDirectory = %s, outputName = %s, sampleRate = %g, "
         "maxPending = %d).\n",
         frameDirectory.c_str(), outputDirectory.c_str(), outputName.c_str(), sampleRate, maxPending);
  if (!writer_.joinable()) writer_ = std::thread(&AsyncVTK::writerLoop, this);
  std::cout << "Serializer Initialized." << std::endl;
}

std::string AsyncVTK::saveState(Job* job) {
  std::cerr << "NOT IMPLEMENTED! Oops." << std::endl;
  return "error";
}

int AsyncVTK::loadState(Job* job, std::string fullpath) {
  std::cerr << "NOT IMPLEMENTED! Oops." << std::endl;
  return 0;
}

namespace {

std::string frame_file(const char* prefix, const Body* body, int frame) {
  std::stringstream ss;
  ss << prefix << "." << body->id << "." << body->name << "." << std::setw(10) << std::setfill('0') << frame << ".vtk";
  return ss.str();
}

std::vector<int> active_flags(const Eigen::VectorXi& a) {
  std::vector<int> out((size_t)a.rows());
  for (int i = 0; i < (int)a.rows(); i++) out[(size_t)i] = a(i);
  return out;
}

}  // namespace

// DefaultVTK::writeFrame (default_vtk.cpp:120-200): the frame condition, the
// two files per body, the title lines (the node file's carries the frame
// count, the point file's the frame index) and the order in which the
// objects write. Everything is captured here and written by the writer
// thread.
int AsyncVTK::writeFrame(Job* job) {
  if (!((job->t - job->t0) >= (sampledFrames / sampleRate) || sampledFrames == 0)) return 0;
  sampledFrames += 1;
  const int index = sampledFrames - 1;
  if (headers_.size() < job->bodies.size()) headers_.resize(job->bodies.size());
  std::vector<std::unique_ptr<Frame>> frame;
  for (size_t b = 0; b < job->bodies.size(); b++) {
    Body* body = job->bodies[b].get();
    std::unique_ptr<Frame> f(new Frame());
    f->ppath = frameDirectory + frame_file("fpd", body, index);
    f->npath = frameDirectory + frame_file("fnd", body, index);
    f->plen = body->points->x.size();
    f->nlen = body->nodes->x.size();
    f->pactive = active_flags(body->points->active);
    f->nactive = active_flags(body->nodes->active);
    current_ = f.get();
    pcap_ << "# vtk DataFile Version 3.0\n";
    pcap_ << "Frame: " << index << ", Time: " << job->t << "\n";
    body->points->writeHeader(job, body, this, pcap_, VTK);
    ncap_ << "# vtk DataFile Version 3.0\n";
    ncap_ << "Frame: " << sampledFrames << ", Time: " << job->t << "\n";
    nodeHeader(job, body, b);
    if (job->activeBodies[b] != 0) {
      body->points->writeFrame(job, body, this);
      body->nodes->writeFrame(job, body, this);
      if (body->activeMaterial != 0) body->material->writeFrame(job, body, this);
      if (body->activeBoundary != 0) body->boundary->writeFrame(job, body, this);
      job->grid->writeFrame(job, this);
    }
    for (size_t c = 0; c < job->contacts.size(); c++) job->contacts[c]->writeFrame(job, this);
    takeText(0);
    takeText(1);
    current_ = nullptr;
    frame.push_back(std::move(f));
  }
  // a writer even when init was skipped, so that the wait below always ends
  if (!writer_.joinable()) writer_ = std::thread(&AsyncVTK::writerLoop, this);
  std::unique_lock<std::mutex> lock(mu_);
  cv_.wait(lock, [&] { return (int)queue_.size() + busy_ < std::max(maxPending, 1); });
  queue_.push_back(std::move(frame));
  lock.unlock();
  cv_.notify_all();
  return 1;
}

// Moves the text collected for one file into the current frame, so that it
// keeps its place among the captured blocks.
void AsyncVTK::takeText(int file) {
  std::stringbuf& buf = file == 0 ? pbuf_ : nbuf_;
  std::string text = buf.str();
  if (text.empty()) return;
  buf.str(std::string());
  Block blk;
  blk.kind = Block::kText;
  blk.file = file;
  blk.text = std::make_shared<const std::string>(std::move(text));
  current_->blocks.push_back(std::move(blk));
}

// The grid's node header (Grid::writeHeader, cartesian.cpp:459-520): reused
// while the body's node positions and active flags are those it was written
// from, else written again into memory and kept.
void AsyncVTK::nodeHeader(Job* job, Body* body, size_t b) {
  takeText(1);
  HeaderCache& hc = headers_[b];
  Nodes* nodes = body->nodes.get();
  const int n = nodes->x.size();
  std::vector<double> x(3 * (size_t)n);
  for (int i = 0; i < n; i++)
    for (int pos = 0; pos < 3; pos++) x[3 * (size_t)i + pos] = nodes->x(i, pos);
  const std::vector<int>& active = current_->nactive;
  if (hc.text && hc.x == x && hc.active == active) {
    Block blk;
    blk.kind = Block::kText;
    blk.file = 1;
    blk.text = hc.text;
    current_->blocks.push_back(std::move(blk));
    return;
  }
  headerCaptured_ = false;
  const size_t before = current_->blocks.size();
  job->grid->writeHeader(job, body, this, ncap_, VTK);
  const bool plain = !headerCaptured_ && current_->blocks.size() == before;
  takeText(1);
  hc.text.reset();
  if (plain && current_->blocks.size() == before + 1) {
    hc.x = std::move(x);
    hc.active = active;
    hc.text = current_->blocks.back().text;
  }
}

void AsyncVTK::flush() {
  std::unique_lock<std::mutex> lock(mu_);
  cv_.wait(lock, [&] { return queue_.empty() && busy_ == 0; });
}

// ---- capture (writeFrame's thread) ----

void AsyncVTK::writeDefaultPointHeader(Job* job, Body* body, std::ofstream& pfile, int SPEC) {
  if (!current_) return;
  takeText(0);
  Block blk;
  blk.kind = Block::kPointHeader;
  blk.dim = body->points->x.DIM;
  blk.count = body->points->x.size();
  blk.values.assign(3 * (size_t)blk.count, 0.0);
  for (int i = 0; i < blk.count; i++)
    for (int pos = 0; pos < blk.dim && pos < 3; pos++) blk.values[3 * (size_t)i + pos] = body->points->x(i, pos);
  current_->blocks.push_back(std::move(blk));
}

void AsyncVTK::writeDefaultNodeHeader(Job* job, Body* body, std::ofstream& nfile, int SPEC) {
  if (!current_) return;
  takeText(1);
  headerCaptured_ = true;
  Block blk;
  blk.kind = Block::kNodeHeader;
  blk.dim = body->nodes->x.DIM;
  blk.count = body->nodes->x.size();
  blk.values.assign(3 * (size_t)blk.count, 0.0);
  for (int i = 0; i < blk.count; i++)
    for (int pos = 0; pos < blk.dim && pos < 3; pos++) blk.values[3 * (size_t)i + pos] = body->nodes->x(i, pos);
  current_->blocks.push_back(std::move(blk));
}

void AsyncVTK::writeScalarArray(Eigen::VectorXd& scalarArray, std::string name) {
  if (!current_) return;
  takeText(0);
  takeText(1);
  Block blk;
  blk.kind = Block::kScalar;
  blk.name = name;
  blk.count = (int)scalarArray.rows();
  blk.values.resize((size_t)blk.count);
  for (int i = 0; i < blk.count; i++) blk.values[(size_t)i] = scalarArray(i);
  current_->blocks.push_back(std::move(blk));
}

void AsyncVTK::writeVectorArray(MPMVectorArray& vectorArray, std::string name) {
  if (!current_) return;
  takeText(0);
  takeText(1);
  Block blk;
  blk.kind = Block::kVector;
  blk.name = name;
  blk.count = vectorArray.size();
  blk.values.resize(3 * (size_t)blk.count);
  for (int i = 0; i < blk.count; i++)
    for (int pos = 0; pos < 3; pos++) blk.values[3 * (size_t)i + pos] = vectorArray(i, pos);
  current_->blocks.push_back(std::move(blk));
}

void AsyncVTK::writeTensorArray(MPMTensorArray& tensorArray, std::string name) {
  if (!current_) return;
  takeText(0);
  takeText(1);
  Block blk;
  blk.kind = Block::kTensor;
  blk.name = name;
  blk.count = tensorArray.size();
  blk.values.resize(9 * (size_t)blk.count);
  for (int i = 0; i < blk.count; i++)
    for (int pos = 0; pos < 9; pos++) blk.values[9 * (size_t)i + pos] = tensorArray(i, pos);
  current_->blocks.push_back(std::move(blk));
}

// ---- formatting (writer thread) ----

void AsyncVTK::writerLoop() {
  for (;;) {
    std::vector<std::unique_ptr<Frame>> frame;
    {
      std::unique_lock<std::mutex> lock(mu_);
      cv_.wait(lock, [&] { return stop_ || !queue_.empty(); });
      if (queue_.empty()) return;
      frame = std::move(queue_.front());
      queue_.pop_front();
      busy_++;
    }
    for (auto& f : frame) format(*f);
    frame.clear();
    {
      std::lock_guard<std::mutex> lock(mu_);
      busy_--;
    }
    cv_.notify_all();
  }
}

namespace {

// Text of the frames. DefaultVTK streams each number with the stream's
// default formatting, which is printf's %g at the stream's precision, 6
// (num_put), in the C locale; snprintf with "%.6g" gives the same
// characters. Large arrays are formatted in chunks on several threads and
// written in order.
void put_num(std::string& s, double v) {
  char buf[32];
  const int k = std::snprintf(buf, sizeof(buf), "%.6g", v);
  s.append(buf, (size_t)k);
}

void put_int(std::string& s, long v) {
  char buf[24];
  const int k = std::snprintf(buf, sizeof(buf), "%ld", v);
  s.append(buf, (size_t)k);
}

// Formats entries [0, n) with `one(text, i)` into `out`, on up to 8 threads
// for large arrays (chunks written in entry order).
template <typename F>
void emit(std::ofstream& out, int n, F one) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int chunks = n < 65536 ? 1 : (int)std::min(hw, 8u);
  std::vector<std::string> text((size_t)chunks);
  auto run = [&](int c) {
    const int b = (int)((int64_t)n * c / chunks), e = (int)((int64_t)n * (c + 1) / chunks);
    std::string& t = text[(size_t)c];
    t.reserve((size_t)(e - b) * 16);
    for (int i = b; i < e; i++) one(t, i);
  };
  std::vector<std::thread> pool;
  for (int c = 1; c < chunks; c++) pool.emplace_back(run, c);
  run(0);
  for (auto& th : pool) th.join();
  for (const std::string& t : text) out.write(t.data(), (std::streamsize)t.size());
}

// The rules of DefaultVTK's writers (default_vtk.cpp): the header writes a
// position component when the axis exists, the entry is active (!= 0) and
// the value finite; scalar and vector arrays write a value when the entry's
// flag is exactly 1 and the value finite; a point tensor is written when the
// point is active and all 9 components are finite, a node tensor (written
// three times per node, as the reference does) when its components are
// finite. Everything else is written as 0.
void header(std::ofstream& out, const AsyncVTK::Block& blk, const std::vector<int>& active) {
  const int n = blk.count;
  out << "ASCII\n";
  out << "DATASET UNSTRUCTURED_GRID\n";
  out << "POINTS " << n << " double\n";
  emit(out, n, [&](std::string& t, int i) {
    for (int pos = 0; pos < 3; pos++) {
      const double v = blk.values[3 * (size_t)i + pos];
      if (pos < blk.dim && active[(size_t)i] != 0 && std::isfinite(v)) {
        put_num(t, v);
        t += ' ';
      } else {
        t += "0 ";
      }
    }
    t += '\n';
  });
  out << "CELLS " << n << " " << 2 * n << "\n";
  emit(out, n, [&](std::string& t, int i) {
    t += "1 ";
    put_int(t, i);
    t += '\n';
  });
  out << "CELL_TYPES " << n << "\n";
  emit(out, n, [&](std::string& t, int) { t += "1\n"; });
  out << "POINT_DATA " << n << "\n";
}

void scalars(std::ofstream& out, const AsyncVTK::Block& blk, const std::vector<int>& active) {
  out << "SCALARS " << blk.name << " double 1\n";
  out << "LOOKUP_TABLE default\n";
  emit(out, blk.count, [&](std::string& t, int i) {
    const double v = blk.values[(size_t)i];
    if (active[(size_t)i] == 1 && std::isfinite(v)) {
      put_num(t, v);
      t += '\n';
    } else {
      t += "0\n";
    }
  });
}

void vectors(std::ofstream& out, const AsyncVTK::Block& blk, const std::vector<int>& active) {
  out << "VECTORS " << blk.name << " double\n";
  emit(out, blk.count, [&](std::string& t, int i) {
    for (int pos = 0; pos < 3; pos++) {
      const double v = blk.values[3 * (size_t)i + pos];
      if (active[(size_t)i] == 1 && std::isfinite(v)) {
        put_num(t, v);
        t += ' ';
      } else {
        t += "0 ";
      }
    }
    t += '\n';
  });
}

void tensor_rows(std::string& t, const double* v, bool write) {
  if (!write) {
    t += "0 0 0\n0 0 0\n0 0 0\n\n";
    return;
  }
  for (int r = 0; r < 3; r++) {
    put_num(t, v[3 * r]);
    t += ' ';
    put_num(t, v[3 * r + 1]);
    t += ' ';
    put_num(t, v[3 * r + 2]);
    t += '\n';
  }
  t += '\n';
}

bool all_finite(const double* t) {
  for (int k = 0; k < 9; k++)
    if (!std::isfinite(t[k])) return false;
  return true;
}

void point_tensors(std::ofstream& out, const AsyncVTK::Block& blk, const std::vector<int>& active) {
  out << "TENSORS " << blk.name << " double\n";
  emit(out, blk.count, [&](std::string& t, int i) {
    const double* v = blk.values.data() + 9 * (size_t)i;
    tensor_rows(t, v, active[(size_t)i] != 0 && all_finite(v));
  });
}

void node_tensors(std::ofstream& out, const AsyncVTK::Block& blk) {
  out << "TENSORS " << blk.name << " double\n";
  emit(out, blk.count, [&](std::string& t, int i) {
    const double* v = blk.values.data() + 9 * (size_t)i;
    const bool finite = all_finite(v);
    for (int rep = 0; rep < 3; rep++) tensor_rows(t, v, finite);
  });
}

}  // namespace

void AsyncVTK::format(Frame& f) {
  std::ofstream pfile(f.ppath, std::ios::trunc), nfile(f.npath, std::ios::trunc);
  const bool p = pfile.is_open(), n = nfile.is_open();
  if (!p) std::cerr << "Could not open point frame: " << f.ppath << " !" << std::endl;
  if (!n) std::cerr << "Could not open node frame: " << f.npath << " !" << std::endl;
  for (const Block& blk : f.blocks) {
    switch (blk.kind) {
      case Block::kText:
        if (blk.file == 0 && p) pfile << *blk.text;
        if (blk.file == 1 && n) nfile << *blk.text;
        break;
      case Block::kPointHeader:
        if (p) header(pfile, blk, f.pactive);
        break;
      case Block::kNodeHeader:
        if (n) header(nfile, blk, f.nactive);
        break;
      case Block::kScalar:
        if (p && blk.count == f.plen) scalars(pfile, blk, f.pactive);
        if (n && blk.count == f.nlen) scalars(nfile, blk, f.nactive);
        break;
      case Block::kVector:
        if (p && blk.count == f.plen) vectors(pfile, blk, f.pactive);
        if (n && blk.count == f.nlen) vectors(nfile, blk, f.nactive);
        break;
      case Block::kTensor:
        if (p && blk.count == f.plen) point_tensors(pfile, blk, f.pactive);
        if (n && blk.count == f.nlen) node_tensors(nfile, blk);
        break;
    }
  }
}
