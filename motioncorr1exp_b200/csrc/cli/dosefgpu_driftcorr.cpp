// dosefgpu_driftcorr: command-line drop-in for the reference program of the
// same name (src-1125/dosefgpu_driftcorr.cpp).  Same flags, defaults,
// clamping, abort messages, default output names, parameter log and
// alignment log lines; the alignment itself runs in libmc (include/mc.h).
#include <sys/stat.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mc.h"
#include "mrc_file.h"

namespace {

struct Options {
  mc_params p;
  float xscale = 1.f, yscale = 1.f;  // -scx -scy
  int nEndSum2 = 0;                  // -2es
  int bSaveSubAreaCorrSum = 0, bSaveRawSum = 0, bSaveStackCorr = 0, bSaveCCmap = 0;
  int bSaveLog = 1, bLogFSC = 0;
  bool bSaveDisp = true;
  int cdx = 0, cdy = 0;
  std::string fnStack, fnRawsum, fnAlignsum, fnAlignsum2, fnStackCorr, fnCCmap, fnLog, fnDark, fnNorm;
  std::string dispRawFFT, dispCorrSum, dispCorrFFT;
};

Options* g_opt = nullptr;

// TextOutput (DFAlign.cu:59-71): stdout plus an append to the log file.
void text_output(const char* s) {
  printf("%s", s);
  if (g_opt && g_opt->bSaveLog) {
    FILE* fp = fopen(g_opt->fnLog.c_str(), "a");
    if (fp) {
      fprintf(fp, "%s", s);
      fclose(fp);
    }
  }
}

// Library log lines; held back while a run is in flight so that the lines of
// the extra outputs (-srs, -2es) can be placed where the reference prints them.
bool g_hold = false;
std::vector<std::string> g_held;

// The mode the "Input Stack" line names: the reference prints the stack
// object's header mode, 7199 for TIFF (mrct.cpp:106), while the plan decodes
// TIFF words as MC_MODE_U8 or 6.
int g_file_mode = -1;

void log_cb(const char* text, void*) {
  std::string line = text;
  int nx, ny, nz, mode;
  if (g_file_mode >= 0 && std::sscanf(text, "Input Stack: Nx(%d) Ny(%d) Nz(%d) Mode(%d)", &nx, &ny, &nz, &mode) == 4) {
    char b[160];
    std::snprintf(b, sizeof(b), "Input Stack: Nx(%d) Ny(%d) Nz(%d) Mode(%d)\n\n", nx, ny, nz, g_file_mode);
    line = b;
  }
  if (g_hold) g_held.push_back(line);
  else text_output(line.c_str());
}

bool starts_with(const std::string& s, const char* p) { return s.compare(0, std::strlen(p), p) == 0; }

// Message (DFAlign.cu:51-54)
void message(const char* s) { printf("%s\n", s); }

void usage() {
  printf("Dose Fractionation Tool:\n");
  printf("Drift correction\n\n");
  printf("    Input: InputStack.mrc [OPTION VALUE] ...\n");
  printf("          *Note: If not specify OPTION, the default value will be used.\n\n");
  printf("           OPTION     VALUE(Default)    Introduction  \n");
  printf("           -crx       0                 Image crop offset X\n");
  printf("           -cry       0                 Image crop offset Y\n");
  printf("           -crd       0                 Image crop dimension. If 0, use maximum size.\n");
  printf("           -cdx/-cdy  0                 Crop dimension X/Y (square: the smaller is used).\n");
  printf("           -bin       1.0               Float number between 1x and 2x. Bin stack before processing.\n");
  printf("           -scx       1.0               Float number (>=1.0). Stretch image along X axis.\n");
  printf("           -scy       1.0               Float number (>=1.0). Stretch image along Y axis.\n");
  printf("           -nst       0                 First frame (0-base) used in alignment.\n");
  printf("           -ned       0                 Last frame (0-base) used in alignment. If 0, use maximum value.\n");
  printf("           -nss       0                 First frame (0-base) used for final sum.\n");
  printf("           -nes       0                 Last frame (0-base) used for final sum. If 0,use maximum value.\n");
  printf("           -2es       0                 Last frame (0-base) used for the second sum.\n");
  printf("           -gpu       0                 GPU device ID.\n");
  printf("           -bft       150               BFactor in pix^2.\n");
  printf("           -pbx       96                Box dimension for searching CC peak.\n");
  printf("           -fod       2                 Number of frame offset for frame comparision.\n");
  printf("           -nps       0                 Radius of noise peak.\n");
  printf("           -kit       1.0               Threshold of alignment error in pixel.\n");
  printf("           -sub       0                 1: Save as sub-area corrected sum. 0: Not. \n");
  printf("           -srs       0                 1: Save uncorrected sum. 0: Not.\n");
  printf("           -ssc       0                 1: Save aligned stack. 0: Not.\n");
  printf("           -scc       0                 1: Save CC Map. 0: Not.\n");
  printf("           -slg       1                 1: Save Log. 0: Not.\n");
  printf("           -atm       1                 1: Align to middle frame. 0: Not.\n");
  printf("           -dsp       1                 1: Save quick results. 0: Not.\n");
  printf("           -fsc       0                 1: Calculate and log FSC. 0: Not.\n");
  printf("           -frs       FileName.mrc      Uncorrected sum\n");
  printf("           -fcs       FileName.mrc      Corrected sum\n");
  printf("           -2cs       FileName.mrc      Corrected second sum\n");
  printf("           -fct       FileName.mrc      Corrected stack\n");
  printf("           -fcm       FileName.mrc      CC map\n");
  printf("           -flg       FileName.txt      Log file\n");
  printf("           -fdk       FileName.mrc      Dark reference\n");
  printf("           -fnm       FileName.mrc      Gain reference\n");
  printf("           -itr       0                 Number of iteration for iterative alignment\n");
  printf("           -ith       0.0               Convergence threshold for iterative alignment (RMSD shift)\n");
  printf("           -ref       0                 1: gradient refinement of the sub-pixel shifts. 0: Not.\n");
}

// getNFrame (DFAlign.cu:344-368).  The reference tries MRC first, so a
// gzip file whose name contains "mrc" is read as a raw MRC header there;
// here the stack is opened in the alignment thread's order (TIFF, MRC-gz,
// MRC) so the frame count is the file's.
int stack_nframe(const std::string& fn) {
  const char* f = fn.c_str();
  if (!starts_with_tiff(f) && !starts_with_gzip(f)) is_mrc(f, false);  // its MRC2000 line
  mc_stack* s = nullptr;
  if (mc_stack_open(f, &s) != MC_OK) return 0;
  mc_stack_info si;
  mc_stack_get_info(s, &si);
  mc_stack_close(s);
  return si.nz;
}

// VerifyPara (dosefgpu_driftcorr.cpp:60-118)
bool verify_para(Options& o) {
  const int nFrame = stack_nframe(o.fnStack);
  if (nFrame <= 1) {
    printf("Not a stack or wrong file. Abort\n");
    return false;
  }
  mc_params& p = o.p;
  if (p.nStart < 0) p.nStart = 0;
  if (p.nEnd >= nFrame) p.nEnd = nFrame - 1;
  if (p.nEnd <= p.nStart) p.nEnd = nFrame - 1;
  if (p.nStartSum < p.nStart) p.nStartSum = p.nStart;
  if (p.nEndSum > p.nEnd) p.nEndSum = p.nEnd;
  if (p.nEndSum <= p.nStartSum) p.nEndSum = p.nEnd;
  if (o.nEndSum2 > p.nEnd) o.nEndSum2 = p.nEnd;
  if (o.nEndSum2 <= p.nStartSum) o.nEndSum2 = 0;
  if (p.FrameDistOffset >= nFrame / 2 || p.FrameDistOffset < 0) {
    printf("Frame distance offset is too big or less than 0. Abort\n");
    return false;
  }
  if (o.nEndSum2 >= p.nEndSum) {
    printf("Last frame # for the second sum image cannot be larger than or equal to that for the first sum image.\n");
    return false;
  }
  return true;
}

// getPara (dosefgpu_driftcorr.cpp:121-515)
bool get_para(int narg, char* argv[], Options& o) {
  mc_default_params(&o.p);
  mc_params& p = o.p;
  o.fnStack = argv[1];
  if (narg % 2 == 1) {
    printf("Wrong number of arguments. Abort.\n");
    return false;
  }
  bool dRaw = true, dAlign = true, dAlign2 = true, dStack = true, dCC = true, dLog = true;
  for (int i = 2; i < narg; i++) {
    const std::string opt = argv[i];
    auto nexti = [&]() { return atoi(argv[++i]); };
    auto nextf = [&]() { return (float)atof(argv[++i]); };
    auto nexts = [&]() { return std::string(argv[++i]); };
    if (opt == "-crx") { p.crop_offsetx = nexti(); continue; }
    if (opt == "-cry") { p.crop_offsety = nexti(); continue; }
    if (opt == "-crd") { p.crop_nsam = nexti(); continue; }
    if (opt == "-cdx") { o.cdx = nexti(); continue; }
    if (opt == "-cdy") { o.cdy = nexti(); continue; }
    if (opt == "-bin") {
      p.bin = nextf();
      if (p.bin > 2.0001) {
        printf("Larger than maximum binning 2. Set to 2.\n");
        p.bin = 2.0;
      } else if (p.bin < 0.9999) {
        printf("Smaller than minimum binning 1. Set to 1.\n");
        p.bin = 1.0;
      }
      continue;
    }
    if (opt == "-scx") {
      o.xscale = nextf();
      if (o.xscale < 1.0) {
        printf("Stretching factor along X-axis needs to be >=1.0.\n");
        return false;
      }
      continue;
    }
    if (opt == "-scy") {
      o.yscale = nextf();
      if (o.yscale < 1.0) {
        printf("Stretching factor along Y-axis needs to be >=1.0.\n");
        return false;
      }
      continue;
    }
    if (opt == "-nst") { p.nStart = nexti(); continue; }
    if (opt == "-ned") { p.nEnd = nexti(); continue; }
    if (opt == "-nss") { p.nStartSum = nexti(); continue; }
    if (opt == "-nes") { p.nEndSum = nexti(); continue; }
    if (opt == "-2es") { o.nEndSum2 = nexti(); continue; }
    if (opt == "-gpu") { p.GPUNum = nexti(); continue; }
    if (opt == "-bft") { p.bfactor = nextf(); continue; }
    if (opt == "-pbx") { p.CCPeakSearchDim = nexti(); continue; }
    if (opt == "-fod") { p.FrameDistOffset = nexti(); continue; }
    if (opt == "-nps") { p.NoisePeakSize = nexti(); continue; }
    if (opt == "-kit") { p.kiThresh = nextf(); continue; }
    if (opt == "-sub") { o.bSaveSubAreaCorrSum = nexti() != 0; continue; }
    if (opt == "-srs") { o.bSaveRawSum = nexti() != 0; continue; }
    if (opt == "-ssc") { o.bSaveStackCorr = nexti() != 0; continue; }
    if (opt == "-scc") { o.bSaveCCmap = nexti() != 0; continue; }
    if (opt == "-slg") { o.bSaveLog = nexti() != 0; continue; }
    if (opt == "-atm") { p.bAlignToMid = nexti() != 0; continue; }
    if (opt == "-dsp") {
      if (nexti() == 0) o.bSaveDisp = false;
      continue;
    }
    if (opt == "-fsc") { o.bLogFSC = nexti() != 0; continue; }
    if (opt == "-frs") { o.fnRawsum = nexts(); dRaw = false; continue; }
    if (opt == "-fcs") { o.fnAlignsum = nexts(); dAlign = false; continue; }
    if (opt == "-2cs") { o.fnAlignsum2 = nexts(); dAlign2 = false; continue; }
    if (opt == "-fct") { o.fnStackCorr = nexts(); dStack = false; continue; }
    if (opt == "-fcm") { o.fnCCmap = nexts(); dCC = false; continue; }
    if (opt == "-flg") { o.fnLog = nexts(); dLog = false; continue; }
    if (opt == "-fnm") { o.fnNorm = nexts(); continue; }
    if (opt == "-fdk") { o.fnDark = nexts(); continue; }
    if (opt == "-itr") { p.iter = nexti(); continue; }
    if (opt == "-ith") { p.iterthres = nextf(); continue; }
    if (opt == "-ref") { p.refine = nexti(); continue; }
    printf("Undefined option: %s .Abort.\n", argv[i]);
    return false;
  }
  if (o.cdx > 0 || o.cdy > 0) {
    const int d = (o.cdx > 0 && o.cdy > 0) ? std::min(o.cdx, o.cdy) : std::max(o.cdx, o.cdy);
    if (o.cdx > 0 && o.cdy > 0 && o.cdx != o.cdy)
      printf("Warning: square crop only; using -cdx/-cdy %d.\n", d);
    p.crop_nsam = d;
  }
  // default file names (dosefgpu_driftcorr.cpp:433-481)
  std::string fnp = argv[1];
  if (fnp.rfind('.') != std::string::npos) fnp = fnp.substr(0, fnp.rfind('.'));
  if (p.bin > 1.0001) fnp += "_binned";
  std::string path = ".", prefix;
  if (fnp.rfind('/') == std::string::npos) prefix = fnp;
  else prefix = fnp.substr(fnp.rfind('/') + 1);
  if (dRaw) o.fnRawsum = prefix + "_SumRaw.mrc";
  if (dAlign) o.fnAlignsum = prefix + "_SumCorr.mrc";
  if (dAlign2) o.fnAlignsum2 = prefix + "_SumCorr2.mrc";
  if (dStack) o.fnStackCorr = prefix + "_Corrected.mrc";
  if (dCC) o.fnCCmap = prefix + "_CCMap.mrc";
  if (dLog) o.fnLog = prefix + "_Log.txt";
  if (o.bSaveDisp) {
    const std::string d = path + "/dosef_quick/" + prefix;
    o.dispRawFFT = d + "_RawFFT.mrc";
    o.dispCorrSum = d + "_CorrSum.mrc";
    o.dispCorrFFT = d + "_CorrFFT.mrc";
  }
  return verify_para(o);
}

// ShowPara (dosefgpu_driftcorr.cpp:517-579)
void show_para(const Options& o) {
  if (!o.bSaveLog) return;
  FILE* fp = fopen(o.fnLog.c_str(), "w");
  if (!fp) return;
  const mc_params& p = o.p;
  fprintf(fp, "******Parameter List******\n");
  fprintf(fp, "Input:  %s\n", o.fnStack.c_str());
  fprintf(fp, "  -crx  %d\n", p.crop_offsetx);
  fprintf(fp, "  -cry  %d\n", p.crop_offsety);
  fprintf(fp, "  -crd  %d\n", p.crop_nsam);
  fprintf(fp, "  -bin  %f\n", p.bin);
  fprintf(fp, "  -scx  %f\n", o.xscale);
  fprintf(fp, "  -scy  %f\n", o.yscale);
  fprintf(fp, "  -nst  %d\n", p.nStart);
  fprintf(fp, "  -ned  %d\n", p.nEnd);
  fprintf(fp, "  -nss  %d\n", p.nStartSum);
  fprintf(fp, "  -nes  %d\n", p.nEndSum);
  fprintf(fp, "  -2es  %d\n", o.nEndSum2);
  fprintf(fp, "  -gpu  %d\n", p.GPUNum);
  fprintf(fp, "  -bft  %f\n", p.bfactor);
  fprintf(fp, "  -pbx  %d\n", p.CCPeakSearchDim);
  fprintf(fp, "  -fod  %d\n", p.FrameDistOffset);
  fprintf(fp, "  -nps  %d\n", p.NoisePeakSize);
  fprintf(fp, "  -kit  %f\n", p.kiThresh);
  fprintf(fp, "  -sub  %d\n", o.bSaveSubAreaCorrSum);
  fprintf(fp, "  -srs  %d\n", o.bSaveRawSum);
  fprintf(fp, "  -ssc  %d\n", o.bSaveStackCorr);
  fprintf(fp, "  -scc  %d\n", o.bSaveCCmap);
  fprintf(fp, "  -slg  %d\n", o.bSaveLog);
  fprintf(fp, "  -atm  %d\n", p.bAlignToMid);
  fprintf(fp, "  -dsp  %d\n", o.bSaveDisp ? 1 : 0);
  fprintf(fp, "  -fsc  %d\n", o.bLogFSC);
  fprintf(fp, "  -fcs  %s\n", o.fnAlignsum.c_str());
  fprintf(fp, "  -2cs  %s\n", o.fnAlignsum2.c_str());
  if (o.bSaveRawSum) fprintf(fp, "  -frs  %s\n", o.fnRawsum.c_str());
  if (o.bSaveStackCorr) fprintf(fp, "  -fct  %s\n", o.fnStackCorr.c_str());
  if (o.bSaveCCmap) fprintf(fp, "  -fcm  %s\n", o.fnCCmap.c_str());
  if (o.bSaveLog) fprintf(fp, "  -flg  %s\n", o.fnLog.c_str());
  if (o.bSaveDisp) {
    fprintf(fp, "\nQuick results in dosef_quick folder:\n");
    fprintf(fp, "UnCorrected FFT: %s \n", o.dispRawFFT.c_str());
    fprintf(fp, "Corrected Sum:   %s \n", o.dispCorrSum.c_str());
    fprintf(fp, "Corrected FFT:   %s \n", o.dispCorrFFT.c_str());
  }
  if (!o.fnDark.empty()) fprintf(fp, "  -fdk  %s\n", o.fnDark.c_str());
  if (!o.fnNorm.empty()) fprintf(fp, "  -fnm  %s\n", o.fnNorm.c_str());
  fprintf(fp, "  -itr  %d\n", p.iter);
  fprintf(fp, "  -ith  %f\n", p.iterthres);
  fprintf(fp, "******Parameter End******\n\n");
  fclose(fp);
}

// Reads a one- or two-frame reference (DFAlign.cu:614-695).
bool read_ref(const std::string& fn, const char* what, const char* plural, int nx, int ny, std::vector<float>& r1,
              std::vector<float>& r2) {
  char str[1024];
  MrcStack s;
  if (s.open(fn.c_str()) <= 0) {
    snprintf(str, sizeof(str), "Error: Failed to open %s reference %s .", what, fn.c_str());
    message(str);
    return false;
  }
  if (nx != s.header().nx || ny != s.header().ny) {
    snprintf(str, sizeof(str), "Error: Image dimension of %s reference %s differs from image stack .", what,
             fn.c_str());
    message(str);
    return false;
  }
  r1.resize((size_t)nx * ny);
  if (!s.read_frame_float(r1.data(), 0)) {
    snprintf(str, sizeof(str), "Error: Failed to read %s reference %s .", what, fn.c_str());
    message(str);
    return false;
  }
  if (s.header().nz > 1) {
    snprintf(str, sizeof(str), "Processing two %s references.", plural);
    message(str);
    r2.resize((size_t)nx * ny);
    s.read_frame_float(r2.data(), 1);
  } else {
    snprintf(str, sizeof(str), "Processing single %s reference.", plural);
    message(str);
    r2.clear();
  }
  return true;
}

// ThreadFunc_cuAlign (DFAlign.cu:456-1355) around libmc.
int run_align(Options& o) {
  char str[2048];
  const char* fn = o.fnStack.c_str();
  // format detection of RunAlign (DFAlign.cu:470-479)
  mc_stack* stack = nullptr;
  const int orc = mc_stack_open(fn, &stack);
  mc_stack_info h{};
  if (orc == MC_OK) mc_stack_get_info(stack, &h);
  if (orc == MC_OK && h.format == MC_STACK_TIFF) {
    printf("Auto-detected file format: TIFF\n");
  } else if (orc == MC_OK && h.format == MC_STACK_MRCZ) {
    printf("Auto-detected file format: MRC-gz\n");
  } else if (!is_mrc(fn, true)) {
    message(orc == MC_OK ? "Only MRC, MRC-gz, TIFF file formats are supported." : mc_last_error());
    if (stack) mc_stack_close(stack);
    return 1;
  }
  if (orc != MC_OK) {
    snprintf(str, sizeof(str), "Error: Failed to open stack %s . (%s)", fn, mc_last_error());
    message(str);
    return 1;
  }
  struct StackCloser {
    mc_stack* s;
    ~StackCloser() { mc_stack_close(s); }
  } closer{stack};
  g_file_mode = h.file_mode;
  mc_plan* plan = nullptr;
  int rc = mc_plan_create(&o.p, h.nx, h.ny, h.nz, h.mode, &plan);
  if (rc != MC_OK) {
    snprintf(str, sizeof(str), "%s", mc_last_error());
    message(str);
    return 1;
  }
  mc_plan_set_log(plan, log_cb, nullptr);
  if (mc_plan_set_stretch(plan, o.xscale, o.yscale) != MC_OK) {
    message(mc_last_error());
    mc_plan_destroy(plan);
    return 1;
  }
  mc_info info;
  mc_plan_info(plan, &info);
  std::vector<float> dark, dark2, norm, norm2;
  if (!o.fnDark.empty() && !read_ref(o.fnDark, "dark", "dark", h.nx, h.ny, dark, dark2)) {
    mc_plan_destroy(plan);
    return 1;
  }
  if (!o.fnNorm.empty() && !read_ref(o.fnNorm, "gain", "norm", h.nx, h.ny, norm, norm2)) {
    mc_plan_destroy(plan);
    return 1;
  }
  if (!dark.empty() || !norm.empty()) {
    rc = mc_plan_set_refs(plan, dark.empty() ? nullptr : dark.data(), dark2.empty() ? nullptr : dark2.data(),
                          norm.empty() ? nullptr : norm.data(), norm2.empty() ? nullptr : norm2.data());
    if (rc != MC_OK) {
      message(mc_last_error());
      mc_plan_destroy(plan);
      return 1;
    }
  }
  // frames nStart..nEnd, read in chunks and handed to the library
  // frames nStart..nEnd in chunks (TIFF chunks decode on host threads)
  const size_t fb = (size_t)h.nx * h.ny * (h.bits / 8);
  const int chunk = 16;
  std::vector<unsigned char> buf(fb * chunk);
  for (int f = 0; f < info.nframe; f += chunk) {
    const int cnt = std::min(chunk, info.nframe - f);
    int got = 0;
    mc_stack_read_frames(stack, buf.data(), info.nstart + f, cnt, &got);
    for (int k = got; k < cnt; k++) {
      if (mc_stack_read_frames(stack, buf.data() + (size_t)k * fb, info.nstart + f + k, 1, nullptr) == MC_OK)
        continue;
      snprintf(str, sizeof(str), "Error when reading #%03d\n", info.nstart + f + k);
      text_output(str);
      std::memset(buf.data() + (size_t)k * fb, 0, fb);
    }
    rc = mc_plan_load_frames(plan, buf.data(), f, cnt);  // returns once buf may be reused
    if (rc != MC_OK) {
      message(mc_last_error());
      mc_plan_destroy(plan);
      return 1;
    }
  }
  std::vector<float> image((size_t)info.nsam * info.nsam);
  g_hold = true;
  g_held.clear();
  rc = mc_plan_run(plan, image.data());
  g_hold = false;
  auto fail = [&](const char* what) {
    for (const auto& l : g_held) text_output(l.c_str());
    snprintf(str, sizeof(str), "Error: %s (%s)", what, mc_last_error());
    message(str);
    mc_plan_destroy(plan);
    return 1;
  };
  if (rc != MC_OK) return fail(mc_strerror(rc));
  // the sum range and the frame after whose "Add Frame" line the second sum
  // is saved (DFAlign.cu:1115-1122, 1198)
  std::vector<double> sxy((size_t)info.nframe * 2);
  int sfirst = 0, slast = 0;
  mc_plan_get_sum_shifts(plan, sxy.data(), &sfirst, &slast);
  const bool second = o.nEndSum2 > 0 && o.nEndSum2 < o.p.nEndSum;
  int sum2_last = o.nEndSum2 - info.nstart;
  if (sum2_last <= sfirst || sum2_last >= info.nframe) sum2_last = info.nframe - 1;
  if (sum2_last > slast) sum2_last = slast;
  auto sub_name = [&](const std::string& fn) {
    char b2[1024];
    snprintf(b2, sizeof(b2), "%s_ox%d_oy%d_dim%d.mrc", fn.substr(0, fn.size() >= 4 ? fn.size() - 4 : 0).c_str(),
             o.p.crop_offsetx, o.p.crop_offsety, info.nsam_unbin);
    return std::string(b2);
  };
  std::vector<float> extra((size_t)info.nsam * info.nsam);
  std::vector<std::string> raw_lines, sum2_lines;
  // -srs: unaligned sum (DFAlign.cu:851-872)
  if (o.bSaveRawSum) {
    if (mc_plan_raw_sum(plan, extra.data()) != MC_OK) return fail("raw sum");
    MrcHeader rh;
    if (!write_mrc_float(o.fnRawsum.c_str(), extra.data(), info.nsam, info.nsam, 1, &rh)) return fail("write");
    snprintf(str, sizeof(str), "Mean=%f   Min=%f   Max=%f\n", rh.dmean, rh.dmin, rh.dmax);
    raw_lines.push_back(str);
    snprintf(str, sizeof(str), "Save Unaligned Sum to: %s\n", o.fnRawsum.c_str());
    raw_lines.push_back(str);
  }
  // -2es: aligned sum of nStartSum..nEndSum2 (DFAlign.cu:1198-1229)
  if (second) {
    if (mc_plan_sum_to(plan, sum2_last + info.nstart, extra.data()) != MC_OK) return fail("second sum");
    const std::string fn = o.bSaveSubAreaCorrSum ? sub_name(o.fnAlignsum2) : o.fnAlignsum2;
    MrcHeader sh;
    if (!write_mrc_float(fn.c_str(), extra.data(), info.nsam, info.nsam, 1, &sh)) return fail("write");
    snprintf(str, sizeof(str), "Mean=%f   Min=%f   Max=%f\n", sh.dmean, sh.dmin, sh.dmax);
    sum2_lines.push_back(str);
    snprintf(str, sizeof(str), "Save Sum to: %s\n", fn.c_str());
    sum2_lines.push_back(str);
  }
  // -ssc: the aligned frames nStartSum..nEndSum (DFAlign.cu:1104-1113, 1154-1263)
  if (o.bSaveStackCorr) {
    MrcStackWriter w;
    if (!w.open(o.fnStackCorr.c_str(), info.nsam, info.nsam, o.p.nEndSum - o.p.nStartSum + 1))
      return fail("write");
    for (int k = sfirst; k <= slast; k++) {
      if (mc_plan_corrected_frame(plan, k + info.nstart, extra.data()) != MC_OK) return fail("corrected frame");
      if (!w.write_frame(extra.data(), k - sfirst)) return fail("write");
    }
    if (!w.close()) return fail("write");
  }
  // -scc: the pair CC windows, box x box x npairs (DFAlign.cu:882-900, 1094-1099)
  std::vector<std::string> cc_lines;
  if (o.bSaveCCmap) {
    const int box = o.p.CCPeakSearchDim;
    std::vector<float> boxes((size_t)box * box * info.npairs);
    if (mc_plan_get_boxes(plan, boxes.data()) != MC_OK) return fail("CC map");
    if (!write_mrc_float(o.fnCCmap.c_str(), boxes.data(), box, box, info.npairs, nullptr)) return fail("write");
    snprintf(str, sizeof(str), "Save CC map to: %s\n", o.fnCCmap.c_str());
    cc_lines.push_back(str);
  }
  // the held log with the extra lines in the reference's places
  char add2[64];
  snprintf(add2, sizeof(add2), "......Add Frame #%03d ", sum2_last + info.nstart);
  for (size_t i = 0; i < g_held.size(); i++) {
    text_output(g_held[i].c_str());
    const bool last_read = starts_with(g_held[i], "......Read and sum frame") &&
                           (i + 1 == g_held.size() || !starts_with(g_held[i + 1], "......Read and sum frame"));
    if (last_read)
      for (const auto& l : raw_lines) text_output(l.c_str());
    if (second && starts_with(g_held[i], add2))
      for (const auto& l : sum2_lines) text_output(l.c_str());
    const bool last_shift = starts_with(g_held[i], "......Shift of Frame") &&
                            (i + 1 == g_held.size() || !starts_with(g_held[i + 1], "......Shift of Frame"));
    if (last_shift)
      for (const auto& l : cc_lines) text_output(l.c_str());
  }
  g_held.clear();
  // -dsp 1: the three 400 x 400 displays in ./dosef_quick
  // (dosefgpu_driftcorr.cpp:484-512; DFAlign.cu:73-178, 841-849, 1270-1286)
  if (o.bSaveDisp) {
    struct stat st;
    if (stat("dosef_quick", &st) != 0) mkdir("dosef_quick", 0755);
    std::vector<int16_t> disp((size_t)MC_QUICKLOOK_DIM * MC_QUICKLOOK_DIM);
    const std::string* names[3] = {&o.dispRawFFT, &o.dispCorrSum, &o.dispCorrFFT};
    for (int which = 0; which < 3; which++) {
      rc = mc_plan_quicklook(plan, which, disp.data());
      if (rc == MC_OK && write_mrc_short(names[which]->c_str(), disp.data(), MC_QUICKLOOK_DIM, MC_QUICKLOOK_DIM, 1))
        continue;
      snprintf(str, sizeof(str), "Warning: display %s not written (%s)\n", names[which]->c_str(),
               rc == MC_OK ? "write" : mc_last_error());
      text_output(str);
    }
  }
  const std::string fnsum = o.bSaveSubAreaCorrSum ? sub_name(o.fnAlignsum) : o.fnAlignsum;
  MrcHeader oh;
  if (!write_mrc_float(fnsum.c_str(), image.data(), info.nsam, info.nsam, 1, &oh)) {
    snprintf(str, sizeof(str), "Error: Failed to write %s\n", fnsum.c_str());
    text_output(str);
    mc_plan_destroy(plan);
    return 1;
  }
  snprintf(str, sizeof(str), "Mean=%f   Min=%f   Max=%f\n", oh.dmean, oh.dmin, oh.dmax);
  text_output(str);
  snprintf(str, sizeof(str), "Save Sum to: %s\n", fnsum.c_str());
  text_output(str);
  // -fsc (PlotFSC's table, DFAlign.cu:309-319)
  if (o.bLogFSC) {
    std::vector<double> rows;
    int nbox = 0;
    rc = mc_plan_fsc(plan, nullptr, 0, &nbox);
    if (rc == MC_OK) {
      rows.resize((size_t)nbox * 5);
      rc = mc_plan_fsc(plan, rows.data(), nbox, &nbox);
    }
    if (rc == MC_OK) {
      text_output("\nFSC parallel(D) and perpendicular(U) to drift direction:\n");
      text_output("   Nq%       D_Raw       U_Raw       D_Corr       U_Corr\n");
      for (int i = 0; i < nbox; i++) {
        const double* r = rows.data() + (size_t)i * 5;
        snprintf(str, sizeof(str), "%7.2f %12.4f %12.4f %12.4f %12.4f\n", r[0], r[1], r[2], r[3], r[4]);
        text_output(str);
      }
      text_output("\n");
    } else {
      snprintf(str, sizeof(str), "Warning: FSC not computed (%s)\n", mc_last_error());
      text_output(str);
    }
  }
  text_output("Done.\n");
  mc_plan_destroy(plan);
  return 0;
}

}  // namespace

int main(int narg, char* argv[]) {
  if (narg == 1) {
    usage();
    return 0;
  }
  Options o;
  g_opt = &o;
  if (!get_para(narg, argv, o)) {
    printf("Error: Have wrong parameters. Abort!\n");
    return 1;
  }
  show_para(o);
  return run_align(o);
}
