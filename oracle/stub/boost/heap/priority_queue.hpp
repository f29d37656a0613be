/* Empty stand-in: the reference AA.h includes this boost header but uses nothing from it. */
