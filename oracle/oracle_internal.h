// Internal declarations shared by the oracle translation units (test infrastructure only).
#pragma once

#include "oracle.h"
#include "../chaste_b200/csrc/models/lr91.h"
#include "../chaste_b200/csrc/models/tt06.h"

namespace orc {

class TimeStepper {
  public:
    TimeStepper(double start, double end, double dt);
    bool AtEnd() const { return mTime >= mEnd; }
    double Time() const { return mTime; }
    double Next() const { return mNext; }
    double NextStep() const { return mNext - mTime; }
    void Advance();
    unsigned Steps() const { return mSteps; }

  private:
    double CalcNext() const;
    double mStart, mEnd, mDt;
    unsigned mSteps;
    double mTime, mNext, mEps;
};

double stimulus_value(const orc_stimulus* s, double t);

template <class M>
void grl_next(int method, double* y, double stim, double cm, const double* p, double h, bool zero_dv);

template <class M>
void except_voltage(int method, double* y, const double* p, const orc_stimulus* stim,
                    double am_div, double cm, double t0, double t1, double dt);

}  // namespace orc
