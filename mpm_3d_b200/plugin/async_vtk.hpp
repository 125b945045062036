// AsyncVTK: an mpm_3d Serializer plugin that writes DefaultVTK's frames
// (src/objects/serializers/default_vtk.cpp) from a background thread, so that
// the step loop does not wait for the text formatting of a frame.
//
// Its config surface is DefaultVTK's (default_vtk.cpp:25-50):
//
//   serializer { class = "AsyncVTK"  properties = {sampleRate}
//                str-properties = {frameDirectory, outputDirectory, outputName}
//                int-properties = {maxPending} }
//
// and it writes the same files with the same bytes: the frame condition and
// file names of DefaultVTK::writeFrame (120-200), and the number formatting
// and zero rules of its header and array writers (55-125, 204-330). At a
// frame, writeFrame lets the objects write as they do for DefaultVTK, but
// nothing reaches a file on that thread: text an object writes into the
// stream it is given (the title lines, a grid's node header) is collected in
// memory, and the default point and node headers and every array handed to
// writeScalarArray / writeVectorArray / writeTensorArray are copied with the
// active flags they are written against. A writer thread formats and writes
// the frames in order. The grid's header text of a body is kept and reused
// while the body's node positions and active flags are unchanged (a
// CartesianLinear header is all positions and fixed connectivity).
// maxPending (default 2) bounds the frames held in memory: writeFrame waits
// while that many are queued. The destructor writes every queued frame
// before it returns.
#ifndef MPM_B200_ASYNC_VTK_HPP
#define MPM_B200_ASYNC_VTK_HPP

#include <condition_variable>
#include <deque>
#include <fstream>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "mpm_objects.hpp"

class AsyncVTK : public Serializer {
 public:
  AsyncVTK();
  ~AsyncVTK() override;

  std::string frameDirectory, outputDirectory, outputName;
  double sampleRate = 0.0;
  int sampledFrames = 0;
  int maxPending = 2;

  void init(Job* job) override;
  std::string saveState(Job* job) override;
  int loadState(Job* job, std::string fullpath) override;
  int writeFrame(Job* job) override;

  void writeDefaultPointHeader(Job* job, Body* body, std::ofstream& pfile, int SPEC) override;
  void writeDefaultNodeHeader(Job* job, Body* body, std::ofstream& nfile, int SPEC) override;
  void writeScalarArray(Eigen::VectorXd& scalarArray, std::string name) override;
  void writeVectorArray(MPMVectorArray& vectorArray, std::string name) override;
  void writeTensorArray(MPMTensorArray& tensorArray, std::string name) override;

  // Blocks until every queued frame is on disk.
  void flush();

  // One deferred piece of a frame file: text for one of the two files, a
  // default header, or a named array (entries in point or node order).
  struct Block {
    enum Kind { kText, kPointHeader, kNodeHeader, kScalar, kVector, kTensor } kind;
    int file = 0;                             // text: 0 point file, 1 node file
    std::shared_ptr<const std::string> text;  // text
    std::string name;
    int dim = 0;                 // header: the position array's DIM
    int count = 0;               // entries
    std::vector<double> values;  // count * width
  };

  // One body's frame: its two files and what is to be written into them.
  struct Frame {
    std::string ppath, npath;
    int plen = 0, nlen = 0;
    std::vector<int> pactive, nactive;  // the body's active flags at the frame
    std::vector<Block> blocks;          // in the order the objects wrote them
  };

 private:
  // The grid header text of a body and the node state it was written from.
  struct HeaderCache {
    std::vector<double> x;
    std::vector<int> active;
    std::shared_ptr<const std::string> text;
  };

  void takeText(int file);
  void nodeHeader(Job* job, Body* body, size_t b);
  void writerLoop();
  static void format(Frame& f);

  Frame* current_ = nullptr;  // the frame being captured (writeFrame's thread)
  // streams handed to the objects; their text collects in memory
  std::stringbuf pbuf_, nbuf_;
  std::ofstream pcap_, ncap_;
  bool headerCaptured_ = false;  // a default header was captured during a grid header call
  std::vector<HeaderCache> headers_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::vector<std::unique_ptr<Frame>>> queue_;  // one entry per frame: its bodies' files
  int busy_ = 0;  // frames taken by the writer and not yet written
  bool stop_ = false;
  std::thread writer_;
};

#endif  // MPM_B200_ASYNC_VTK_HPP
