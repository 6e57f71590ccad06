"""Inert stand-in for matplotlib (the reference imports it in nonlinear/main3d.py:10-11,
for plots that are switched off by doPlot=False at :15).  Used only by make_golden.py."""
cm = None
def use(*a, **kw):
    pass
