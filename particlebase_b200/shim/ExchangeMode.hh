// Kinds of per-particle arrays exchanged between GPUs (ExchangeMode.hh); kept
// for source compatibility, there is one GPU.
#if !defined(EXCHANGEMODE)
#define EXCHANGEMODE

enum class ExchangeMode { force, acceleration, torque, coordnumber, density };

#endif
