        SampleA                 SampleB                 SampleC
SampleA 0                       0.693834      0.272899
SampleB 0.693834      0                       0.707595
SampleC 0.272899      0.707595      0
